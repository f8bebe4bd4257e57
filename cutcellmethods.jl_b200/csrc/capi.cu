// capi.cu -- the C ABI of libcutcell_b200.so (include/cutcell_b200.h).
//
// Host-side validation mirrors the reference's (DimensionMismatch: src/cache.jl:107-121,
// src/marching_squares/cache.jl:140-147; ArgumentError for an anisotropic PLIC grid:
// src/plic/surface.jl:41-45) and returns status codes the shims turn back into those exceptions.
// The op-tape and tiling table are validated before they reach a kernel, so no device code ever
// indexes outside them.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_internal.h"

namespace {

thread_local std::string g_last_error;

cc_status cuda_fail(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return CC_CUDA_ERR;
}
cc_status fail(cc_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

// Packed tapes: every op gets its own copy of its primitive's parameters, started on a 4-element
// boundary and padded to a multiple of 4 elements (at most 16), plus, for a smooth-min, its k --
// at most 3 + 16 + 1 = 20 slots per op.
constexpr int PACK_MAX_PARAMS = 20 * CC_TAPE_MAX_OPS;
constexpr size_t TAPE_CAP = CC_TAPE_MAX_OPS * sizeof(cc_op) + PACK_MAX_PARAMS * sizeof(double) + 64;

int prim_params(int opcode, int dim) {
  switch (opcode) {
    case CC_OP_NONE: return 0;
    case CC_OP_SPHERE: return dim + 1;
    case CC_OP_BOX: return 2 * dim;
    case CC_OP_TORUS: return dim == 3 ? 14 : -1;
    case CC_OP_PLANE: return 2 * dim;
    case CC_OP_TRIG: return dim + 2;
    case CC_OP_CONST: return 1;
    case CC_OP_STAR: return dim == 2 ? 13 : -1;
    default: return -1;
  }
}

cc_status validate_tape(const cc_optape* t, int dim) {
  if (!t || !t->ops) return fail(CC_BAD_TAPE, "null op-tape");
  if (t->n_ops < 1 || t->n_ops > CC_TAPE_MAX_OPS) return fail(CC_BAD_TAPE, "op-tape length out of range");
  if (t->n_params < 0 || t->n_params > CC_TAPE_MAX_PARAMS || (t->n_params > 0 && !t->params))
    return fail(CC_BAD_TAPE, "op-tape parameter count out of range");
  int sp = 0;
  for (int i = 0; i < t->n_ops; ++i) {
    const cc_op& op = t->ops[i];
    if (op.combine > CC_COMB_NEG) return fail(CC_BAD_TAPE, "unknown combine mode");
    const int np = prim_params(op.opcode, dim);
    if (np < 0) return fail(CC_BAD_TAPE, "primitive not available in this dimension");
    if (op.opcode == CC_OP_NONE) {
      if (op.combine == CC_COMB_NEG) {
        if (sp < 1) return fail(CC_BAD_TAPE, "negate on an empty stack");
        continue;
      }
      if (op.combine == CC_COMB_PUSH) return fail(CC_BAD_TAPE, "pop-and-push op");
      if (sp < 2) return fail(CC_BAD_TAPE, "combinator needs two operands");
      --sp;
    } else {
      if (op.combine == CC_COMB_NEG) return fail(CC_BAD_TAPE, "negate carries no primitive");
      if (int(op.poff) + np > t->n_params) return fail(CC_BAD_TAPE, "primitive parameters out of range");
      if (op.combine == CC_COMB_PUSH) ++sp;
      else if (sp < 1) return fail(CC_BAD_TAPE, "combine into an empty stack");
    }
    if (op.combine == CC_COMB_SMIN) {
      if (op.kparam >= t->n_params) return fail(CC_BAD_TAPE, "smooth-min parameter out of range");
      if (!(t->params[op.kparam] > 0.0)) return fail(CC_BAD_TAPE, "smooth-min k must be positive");
    }
    if (sp > CC_TAPE_MAX_STACK) return fail(CC_BAD_TAPE, "op-tape stack too deep");
  }
  if (sp != 1) return fail(CC_BAD_TAPE, "op-tape does not leave exactly one value");
  return CC_OK;
}

struct DeviceGuard {
  int old = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&old);
    if (old != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (old >= 0 && cur != old) cudaSetDevice(old);
  }
};

}  // namespace

namespace cci {
void set_last_error(const std::string& msg) { g_last_error = msg; }

// Every index a kernel takes from a tiling table blob is checked here, once, on the host: lookup
// entries (test count, Lewiner case, face codes, outcome range), outcomes (interior-test kind,
// edge, tiles) and tiles (triangle count, code range, codes 1..13).
bool check_mc_table(const unsigned char* b, size_t nbytes, TableLayout* out, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (!b) return no("null table");
  if (nbytes < sizeof(cc_mc_table_header) + 256 * sizeof(cc_mc_lut)) return no("table too short");
  cc_mc_table_header hd;
  std::memcpy(&hd, b, sizeof hd);
  if (hd.magic != CC_MC_TABLE_MAGIC || hd.version != 1) return no("not a tiling table");
  const size_t need = sizeof(cc_mc_table_header) + 256 * sizeof(cc_mc_lut) + hd.n_outcomes * sizeof(cc_mc_outcome) +
                      hd.n_tiles * sizeof(cc_mc_tile) + hd.n_codes;
  if (need > nbytes || hd.total_bytes != nbytes || hd.n_outcomes > 65535 || hd.n_tiles > 65535)
    return no("table sizes inconsistent");
  const cc_mc_lut* luts = reinterpret_cast<const cc_mc_lut*>(b + sizeof hd);
  const cc_mc_outcome* outs = reinterpret_cast<const cc_mc_outcome*>(luts + 256);
  const cc_mc_tile* tiles = reinterpret_cast<const cc_mc_tile*>(outs + hd.n_outcomes);
  const uint8_t* codes = reinterpret_cast<const uint8_t*>(tiles + hd.n_tiles);
  for (int l = 0; l < 256; ++l) {
    const cc_mc_lut& e = luts[l];
    if (e.ntests > 6 || e.lcase < 1 || e.lcase > 15) return no("bad lookup entry");
    if (size_t(e.outcome_base) + (size_t(1) << e.ntests) > hd.n_outcomes) return no("outcome out of range");
    for (int i = 0; i < e.ntests; ++i)
      if (e.face[i] == 0 || e.face[i] > 6 || e.face[i] < -6) return no("bad face code");
  }
  for (uint32_t o = 0; o < hd.n_outcomes; ++o) {
    const cc_mc_outcome& oc = outs[o];
    if (oc.itype > CC_MC_INTERIOR_EDGE || oc.edge > 11 || oc.tile_true >= hd.n_tiles || oc.tile_false >= hd.n_tiles)
      return no("bad outcome");
  }
  for (uint32_t t = 0; t < hd.n_tiles; ++t) {
    if (tiles[t].ntris > 16 || size_t(tiles[t].code_off) + 3u * tiles[t].ntris > hd.n_codes) return no("bad tile");
    for (int c = 0; c < 3 * tiles[t].ntris; ++c)
      if (codes[tiles[t].code_off + c] < 1 || codes[tiles[t].code_off + c] > 13) return no("bad edge code");
  }
  if (out) {
    out->n_outcomes = hd.n_outcomes;
    out->n_tiles = hd.n_tiles;
  }
  return true;
}

DevTable TableLayout::at(const unsigned char* dev) const {
  DevTable tb;
  tb.luts = reinterpret_cast<const cc_mc_lut*>(dev + sizeof(cc_mc_table_header));
  tb.outs = reinterpret_cast<const cc_mc_outcome*>(tb.luts + 256);
  tb.tiles = reinterpret_cast<const cc_mc_tile*>(tb.outs + n_outcomes);
  tb.codes = reinterpret_cast<const uint8_t*>(tb.tiles + n_tiles);
  return tb;
}
}  // namespace cci


namespace {

}  // namespace

namespace cci {

// Pack a validated tape for the device into `out` (capacity tape_pack_capacity()): the ops,
// padded to 16 bytes, then each primitive's parameter block moved to a 4-element boundary (read
// there with vector loads), each smooth-min k copied beside the blocks, everything narrowed to T.
// Returns the packed size in bytes; *n_params receives the packed parameter count.
template <class T>
size_t pack_tape(const cc_optape* t, int dim, unsigned char* out, int* n_params) {
  const size_t ops_bytes = ((t->n_ops * sizeof(cc_op) + 15) / 16) * 16;
  cc_op* ops = reinterpret_cast<cc_op*>(out);
  T* p = reinterpret_cast<T*>(out + ops_bytes);
  int np = 0;
  for (int i = 0; i < t->n_ops; ++i) {
    cc_op op = t->ops[i];
    if (op.opcode != CC_OP_NONE) {
      // a primitive's parameters start on a 4-element boundary: the device reads them with
      // vector loads (an SMIN constant before them may have left np unaligned)
      while (np % 4) p[np++] = T(0);
      const int cnt = prim_params(op.opcode, dim);
      const int padded = ((cnt + 3) / 4) * 4;
      for (int q = 0; q < padded; ++q) p[np + q] = q < cnt ? T(t->params[op.poff + q]) : T(0);
      op.poff = uint16_t(np);
      np += padded;
    }
    if (op.combine == CC_COMB_SMIN) {
      p[np] = T(t->params[op.kparam]);
      op.kparam = uint16_t(np);
      np += 1;
    }
    ops[i] = op;
  }
  for (size_t b = t->n_ops * sizeof(cc_op); b < ops_bytes; ++b) out[b] = 0;
  *n_params = np;
  return ops_bytes + np * sizeof(T);
}
// 1 for a union (PUSH then MIN) of spheres, 2 for a smooth union (PUSH then SMIN), else 0.
int tape_prunable(const cc_optape* t) {
  if (t->n_ops < 2 || t->ops[0].combine != CC_COMB_PUSH) return 0;
  const int mode = t->ops[1].combine;
  if (mode != CC_COMB_MIN && mode != CC_COMB_SMIN) return 0;
  for (int i = 0; i < t->n_ops; ++i) {
    if (t->ops[i].opcode != CC_OP_SPHERE) return 0;
    if (i > 0 && t->ops[i].combine != mode) return 0;
  }
  return mode == CC_COMB_MIN ? 1 : 2;
}

// A deeper slab keeps a few more spheres per cell but bounds the union less often. On the 64-sphere
// cloud (radii U[0.02, 0.08]) the Float32 update was fastest at 16 layers at 512^3 (3.27 ms; 8:
// 3.31, 32: 3.50) and at 8 at 256^3 (0.676 ms; 16: 0.696, 4: 0.698): the same thickness in space,
// about 0.6 of the median radius.
int prune_slab(const cc_optape* t, double h) {
  if (!t || t->n_ops < 1 || !(h > 0.0)) return 8;
  std::vector<double> r;
  for (int i = 0; i < t->n_ops; ++i)
    if (t->ops[i].opcode == CC_OP_SPHERE && t->ops[i].poff + 3 < t->n_params)
      r.push_back(std::fabs(t->params[t->ops[i].poff + 3]));  // a 3D sphere: centre, radius
  if (r.empty()) return 8;
  std::nth_element(r.begin(), r.begin() + r.size() / 2, r.end());
  const double want = 0.6 * r[r.size() / 2] / h;
  int best = 4;
  for (int s = 8; s <= 32; s *= 2)
    if (std::fabs(std::log2(want / s)) < std::fabs(std::log2(want / best))) best = s;
  return best;
}

template size_t pack_tape<float>(const cc_optape*, int, unsigned char*, int*);
template size_t pack_tape<double>(const cc_optape*, int, unsigned char*, int*);
size_t tape_pack_capacity() { return TAPE_CAP; }

}  // namespace cci

namespace {

// Pack a validated tape and upload it into the handle's buffer, ordered on stream s.
template <class T>
cc_status upload_tape(cc_handle* h, const cc_optape* t, int dim, cudaStream_t s, cci::DevTape* out) {
  if (h->tape_pending) {
    const cudaError_t e = cudaEventSynchronize(h->tape_copied);
    if (e != cudaSuccess) return cuda_fail(e, "tape staging");
    h->tape_pending = false;
  }
  int np = 0;
  const size_t bytes = cci::pack_tape<T>(t, dim, h->tape_host, &np);
  cudaError_t e = cudaMemcpyAsync(h->tape_dev, h->tape_host, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "tape upload");
  e = cudaEventRecord(h->tape_copied, s);
  if (e != cudaSuccess) return cuda_fail(e, "tape upload");
  h->tape_pending = true;
  out->bytes = h->tape_dev;
  out->n_ops = t->n_ops;
  out->n_params = np;
  out->bytes_len = int(bytes);
  out->prunable = cci::tape_prunable(t);
  return CC_OK;
}

template <class T>
cci::DevGrid<T> dev_grid(const cc_grid* g) {
  cci::DevGrid<T> d;
  for (int a = 0; a < 3; ++a) {
    d.x0[a] = T(g->x0[a]);
    d.d[a] = T(g->d[a]);
    d.n[a] = g->n[a];
  }
  if (g->dim == 2) d.n[2] = 1;
  return d;
}

cci::Cols cols_of(const cc_cells* c) {
  cci::Cols k;
  k.kind = c->kind;
  k.amb = c->ambiguous;
  k.vf = c->volume_fraction;
  k.c = c->centroid;
  k.ff = c->face_fraction;
  k.fcl = c->face_centroid_local;
  k.ic = c->interface_centroid;
  return k;
}

bool cells_complete(const cc_cells* c) {
  return c && c->kind && c->ambiguous && c->volume_fraction && c->centroid && c->face_fraction &&
         c->face_centroid_local && c->interface_centroid;
}

cc_status check_grid(const cc_handle* h, const cc_grid* g, int method) {
  if (!h) return fail(CC_BAD_ARG, "null handle");
  if (!g) return fail(CC_BAD_ARG, "null grid");
  if (h->method != method) return fail(CC_BAD_ARG, "handle was created for another method");
  if (h->tree) return fail(CC_BAD_ARG, "a tree-layout cache is updated over its tree, not a grid");
  if (g->dim != h->dim) return fail(CC_DIM_MISMATCH, "grid dimension differs from the cache's");
  for (int a = 0; a < g->dim; ++a) {
    if (g->n[a] != h->n[a]) {
      char buf[256];
      std::snprintf(buf, sizeof buf,
                    "the cache holds %lld cells along axis %d, but `grid` has %lld; a cache is allocated "
                    "for one grid's `n`, and only its origin may move between updates",
                    (long long)h->n[a], a + 1, (long long)g->n[a]);
      return fail(CC_DIM_MISMATCH, buf);
    }
    if (!(g->d[a] > 0.0)) return fail(CC_BAD_ARG, "cell size must be positive");
  }
  return CC_OK;
}

bool isotropic(const cc_grid* g) {
  for (int a = 1; a < g->dim; ++a)
    if (g->d[a] != g->d[0]) return false;
  return true;
}

}  // namespace

namespace cci {
cc_status validate_body(const cc_optape* t, int dim) { return validate_tape(t, dim); }

void* prune_scratch(cc_handle* h, size_t bytes) {
  if (bytes <= h->prune_bytes) return h->prune;
  if (h->prune) cudaFree(h->prune);
  h->prune = nullptr;
  h->prune_bytes = 0;
  if (cudaMalloc(&h->prune, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  h->prune_bytes = bytes;
  return h->prune;
}
cc_status upload_body_f64(cc_handle* h, const cc_optape* t, int dim, cudaStream_t s, DevTape* out) {
  return upload_tape<double>(h, t, dim, s, out);
}
cc_status upload_body_f32(cc_handle* h, const cc_optape* t, int dim, cudaStream_t s, DevTape* out) {
  return upload_tape<float>(h, t, dim, s, out);
}
}  // namespace cci

extern "C" {

const char* cc_version(void) { return "cutcell_b200 0.1.0 (sm_100a)"; }
const char* cc_last_error(void) { return g_last_error.c_str(); }

int64_t cc_set_wait_limit(int64_t polls) { return cci::set_wait_limit(polls); }

cc_status cc_handle_create(int32_t device, int32_t method, int32_t dim, int32_t prec, const int64_t n[3],
                           cc_handle** out) {
  if (!out || !n) return fail(CC_BAD_ARG, "null argument");
  *out = nullptr;
  if (method < CC_MARCHING_SQUARES || method > CC_PLIC) return fail(CC_BAD_ARG, "unknown method");
  if (dim != 2 && dim != 3) return fail(CC_BAD_ARG, "dimension must be 2 or 3");
  if (method == CC_MARCHING_SQUARES && dim != 2) return fail(CC_BAD_ARG, "marching squares is 2D");
  if (method == CC_MARCHING_CUBES && dim != 3) return fail(CC_BAD_ARG, "marching cubes is 3D");
  if (prec != CC_F32 && prec != CC_F64 && prec != CC_MIXED) return fail(CC_BAD_ARG, "unsupported precision");
  const bool tree = method == CC_MARCHING_SQUARES && n[1] == 0;
  for (int a = 0; a < (tree ? 1 : dim); ++a)
    if (n[a] < 1) return fail(CC_BAD_ARG, "every axis needs at least one cell");
  if (method == CC_MARCHING_CUBES && double(n[0]) * double(n[1]) * double(n[2]) > 4294967295.0)
    return fail(CC_TOO_LARGE, "marching cubes indexes at most 2^32 - 1 cells per cache");
  DeviceGuard dg(device);
  cc_handle* h = new cc_handle();
  h->device = device;
  h->method = method;
  h->dim = dim;
  h->prec = prec;
  h->tree = tree;
  for (int a = 0; a < 3; ++a) h->n[a] = a < dim ? n[a] : 1;
  if (tree) { h->n[1] = 0; h->n[2] = 0; }
  cudaError_t e = cudaMalloc(&h->tape_dev, TAPE_CAP);
  if (e == cudaSuccess) e = cudaMallocHost(&h->tape_host, TAPE_CAP);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->tape_copied, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&h->vol_scratch, (2 * cci::calc_volume_blocks() + 2) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&h->rep_scratch, 8 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost(&h->rep_host, 8 * sizeof(unsigned long long));

  if (e == cudaSuccess && method == CC_MARCHING_CUBES) {
    const int64_t ncell = h->n[0] * h->n[1] * h->n[2];
    e = cudaMalloc(&h->cut_list, size_t(ncell) * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&h->cut_count, sizeof(unsigned));
  }
  if (e == cudaSuccess && method == CC_PLIC && dim == 3 && !tree)
    e = cudaMalloc(&h->plic_sides, size_t(h->n[0] * h->n[1] * h->n[2]));
  if (e != cudaSuccess) {
    cc_handle_destroy(h);
    return cuda_fail(e, "cc_handle_create");
  }
  *out = h;
  return CC_OK;
}

cc_status cc_handle_destroy(cc_handle* h) {
  if (!h) return CC_OK;
  DeviceGuard dg(h->device);
  if (h->tape_copied) { cudaEventSynchronize(h->tape_copied); cudaEventDestroy(h->tape_copied); }
  if (h->tape_dev) cudaFree(h->tape_dev);
  if (h->tape_host) cudaFreeHost(h->tape_host);
  if (h->table_dev) cudaFree(h->table_dev);
  if (h->vol_scratch) cudaFree(h->vol_scratch);
  if (h->rep_scratch) cudaFree(h->rep_scratch);
  if (h->rep_host) cudaFreeHost(h->rep_host);
  if (h->cut_list) cudaFree(h->cut_list);
  if (h->cut_count) cudaFree(h->cut_count);
  if (h->plic_sides) cudaFree(h->plic_sides);
  if (h->mesh_vbase) cudaFree(h->mesh_vbase);
  if (h->mesh_scan) cudaFree(h->mesh_scan);
  if (h->mesh_list) cudaFree(h->mesh_list);
  if (h->prune) cudaFree(h->prune);
  cci::free_ms_mesh(h);
  cci::free_plic_mesh(h);
  delete h;
  return CC_OK;
}

cc_status cc_handle_set_mc_table(cc_handle* h, const void* blob, size_t nbytes) {
  if (!h || !blob) return fail(CC_BAD_ARG, "null argument");
  std::string why;
  cci::TableLayout lay;
  if (!cci::check_mc_table(static_cast<const unsigned char*>(blob), nbytes, &lay, &why)) return fail(CC_BAD_TABLE, why);
  DeviceGuard dg(h->device);
  if (h->table_dev) { cudaFree(h->table_dev); h->table_dev = nullptr; }
  cudaError_t e = cudaMalloc(&h->table_dev, nbytes);
  if (e != cudaSuccess) return cuda_fail(e, "table upload");
  e = cudaMemcpy(h->table_dev, blob, nbytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "table upload");
  h->table_bytes = nbytes;
  h->tb = lay.at(h->table_dev);
  return CC_OK;
}

static cc_status mc_common(cc_handle* h, const cc_grid* g, const cc_optape* body, const void* phi_in, void* phi_out,
                           const cc_cells* cells, void* stream) {
  cc_status st = check_grid(h, g, CC_MARCHING_CUBES);
  if (st != CC_OK) return st;
  if (!h->table_dev) return fail(CC_NO_TABLE, "no marching-cubes tiling table set on the handle");
  if (!cells_complete(cells) || (!phi_in && !phi_out)) return fail(CC_BAD_ARG, "null column pointer");
  if (body) {
    st = validate_tape(body, 3);
    if (st != CC_OK) return st;
  }
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cci::DevTape tape{nullptr, 0, 0, 0};
  cudaError_t e;
  ++h->generation;
  if (h->prec == CC_F64) {
    if (body && (st = upload_tape<double>(h, body, 3, s, &tape)) != CC_OK) return st;
    const size_t pb = tape.prunable ? cci::mc_prune_bytes(g->n[0], g->n[1], g->n[2], tape.n_ops, true) : 0;
    void* ps = pb ? cci::prune_scratch(h, pb) : nullptr;
    e = cci::launch_mc<double>(dev_grid<double>(g), tape, static_cast<const double*>(phi_in),
                               static_cast<double*>(phi_out), cols_of(cells), h->tb, h->cut_list, h->cut_count, s,
                               true, false, ps, ps ? pb : 0);
  } else {
    if (body && (st = upload_tape<float>(h, body, 3, s, &tape)) != CC_OK) return st;
    const size_t pb = tape.prunable ? cci::mc_prune_bytes(g->n[0], g->n[1], g->n[2], tape.n_ops, false) : 0;
    void* ps = pb ? cci::prune_scratch(h, pb) : nullptr;
    e = cci::launch_mc<float>(dev_grid<float>(g), tape, static_cast<const float*>(phi_in),
                              static_cast<float*>(phi_out), cols_of(cells), h->tb, h->cut_list, h->cut_count, s, true,
                              h->prec == CC_MIXED, ps, ps ? pb : 0);
  }
  if (e != cudaSuccess) return cuda_fail(e, "marching cubes launch");
  return CC_OK;
}

cc_status cc_mc_update(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi, const cc_cells* cells,
                       void* stream) {
  if (!body) return fail(CC_BAD_TAPE, "null op-tape");
  return mc_common(h, g, body, nullptr, phi, cells, stream);
}

cc_status cc_mc_cells_from_phi(cc_handle* h, const cc_grid* g, const void* phi, const cc_cells* cells, void* stream) {
  if (!phi) return fail(CC_BAD_ARG, "null phi");
  return mc_common(h, g, nullptr, phi, nullptr, cells, stream);
}

static cc_status ms_common(cc_handle* h, const cc_grid* g, const cc_optape* body, const void* phi_in, void* phi_out,
                           const cc_cells* cells, void* stream) {
  cc_status st = check_grid(h, g, CC_MARCHING_SQUARES);
  if (st != CC_OK) return st;
  if (!cells_complete(cells) || (!phi_in && !phi_out)) return fail(CC_BAD_ARG, "null column pointer");
  if (body && (st = validate_tape(body, 2)) != CC_OK) return st;
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cci::DevTape tape{nullptr, 0, 0, 0};
  cudaError_t e;
  if (h->prec == CC_F64) {
    if (body && (st = upload_tape<double>(h, body, 2, s, &tape)) != CC_OK) return st;
    e = cci::launch_ms<double>(dev_grid<double>(g), tape, static_cast<const double*>(phi_in),
                               static_cast<double*>(phi_out), cols_of(cells), s);
  } else {
    if (body && (st = upload_tape<float>(h, body, 2, s, &tape)) != CC_OK) return st;
    e = cci::launch_ms<float>(dev_grid<float>(g), tape, static_cast<const float*>(phi_in),
                              static_cast<float*>(phi_out), cols_of(cells), s, h->prec == CC_MIXED);
  }
  if (e != cudaSuccess) return cuda_fail(e, "marching squares launch");
  return CC_OK;
}

cc_status cc_ms_update(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi, const cc_cells* cells,
                       void* stream) {
  if (!body) return fail(CC_BAD_TAPE, "null op-tape");
  return ms_common(h, g, body, nullptr, phi, cells, stream);
}

cc_status cc_ms_cells_from_phi(cc_handle* h, const cc_grid* g, const void* phi, const cc_cells* cells, void* stream) {
  if (!phi) return fail(CC_BAD_ARG, "null phi");
  return ms_common(h, g, nullptr, phi, nullptr, cells, stream);
}

cc_status cc_ms_tree_update(cc_handle* h, const cc_tree* t, const cc_optape* body, void* phi4, const cc_cells* cells,
                            void* stream) {
  if (!h || !t) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_MARCHING_SQUARES) return fail(CC_BAD_ARG, "handle was created for another method");
  if (!h->tree) return fail(CC_BAD_ARG, "a grid-layout cache is updated over its grid, not a tree");
  if (t->nleaves != h->n[0]) {
    char buf[200];
    std::snprintf(buf, sizeof buf, "the cache holds %lld leaves, but `mesh` has %lld; on an `AdaptiveMesh` both are "
                  "one entry per leaf, in leaf order", (long long)h->n[0], (long long)t->nleaves);
    return fail(CC_DIM_MISMATCH, buf);
  }
  if (!cells_complete(cells) || !phi4 || (t->nleaves > 0 && (!t->level || !t->coord)))
    return fail(CC_BAD_ARG, "null column pointer");
  cc_status st = validate_tape(body, 2);
  if (st != CC_OK) return st;
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cci::DevTape tape{nullptr, 0, 0, 0};
  cudaError_t e;
  if (h->prec == CC_F64) {
    if ((st = upload_tape<double>(h, body, 2, s, &tape)) != CC_OK) return st;
    const double x0[2] = {t->x0[0], t->x0[1]};
    e = cci::launch_ms_tree<double>(x0, t->base_d, t->nleaves, t->level, t->coord, tape, static_cast<double*>(phi4),
                                    cols_of(cells), s);
  } else {
    if ((st = upload_tape<float>(h, body, 2, s, &tape)) != CC_OK) return st;
    const float x0[2] = {float(t->x0[0]), float(t->x0[1])};
    e = cci::launch_ms_tree<float>(x0, t->base_d, t->nleaves, t->level, t->coord, tape, static_cast<float*>(phi4),
                                   cols_of(cells), s, h->prec == CC_MIXED);
  }
  if (e != cudaSuccess) return cuda_fail(e, "tree launch");
  return CC_OK;
}

cc_status cc_plic_update(cc_handle* h, const cc_grid* g, const cc_optape* body, const cc_cells* cells, void* normals,
                         void* intercepts, uint8_t* is_valid, void* stream) {
  cc_status st = check_grid(h, g, CC_PLIC);
  if (st != CC_OK) return st;
  if (!isotropic(g)) return fail(CC_ANISOTROPIC, "PLIC needs an isotropic grid (equal cell size on every axis)");
  if (!cells || !cells->kind || !cells->volume_fraction || !cells->face_fraction || !normals || !intercepts || !is_valid)
    return fail(CC_BAD_ARG, "null column pointer");
  if ((st = validate_tape(body, g->dim)) != CC_OK) return st;
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cci::DevTape tape{nullptr, 0, 0, 0};
  cudaError_t e;
  ++h->generation;
  if (h->prec == CC_F64) {
    if ((st = upload_tape<double>(h, body, g->dim, s, &tape)) != CC_OK) return st;
    tape.slab = g->dim == 3 ? cci::prune_slab(body, g->d[0]) : 8;
    e = g->dim == 3 ? cci::launch_plic<double, 3>(dev_grid<double>(g), tape, cols_of(cells), static_cast<double*>(normals),
                                                  static_cast<double*>(intercepts), is_valid, h->plic_sides, s)
                    : cci::launch_plic<double, 2>(dev_grid<double>(g), tape, cols_of(cells), static_cast<double*>(normals),
                                                  static_cast<double*>(intercepts), is_valid, h->plic_sides, s);
  } else {
    if ((st = upload_tape<float>(h, body, g->dim, s, &tape)) != CC_OK) return st;
    tape.slab = g->dim == 3 ? cci::prune_slab(body, g->d[0]) : 8;
    const bool mx = h->prec == CC_MIXED;
    e = g->dim == 3 ? cci::launch_plic<float, 3>(dev_grid<float>(g), tape, cols_of(cells), static_cast<float*>(normals),
                                                 static_cast<float*>(intercepts), is_valid, h->plic_sides, s, mx)
                    : cci::launch_plic<float, 2>(dev_grid<float>(g), tape, cols_of(cells), static_cast<float*>(normals),
                                                 static_cast<float*>(intercepts), is_valid, h->plic_sides, s, mx);
  }
  if (e != cudaSuccess) return cuda_fail(e, "PLIC launch");
  return CC_OK;
}

cc_status cc_calc_volume(cc_handle* h, const cc_grid* g, const cc_optape* body, double* out, void* stream) {
  if (!h || !g || !out) return fail(CC_BAD_ARG, "null argument");
  if (g->dim != 2 && g->dim != 3) return fail(CC_BAD_ARG, "dimension must be 2 or 3");
  if (!isotropic(g)) return fail(CC_ANISOTROPIC, "calc_volume needs an isotropic grid (equal cell size on every axis)");
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] < 1 || !(g->d[a] > 0.0)) return fail(CC_BAD_ARG, "bad grid");
  cc_status st = validate_tape(body, g->dim);
  if (st != CC_OK) return st;
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  // calc_volume prunes over slabs of 8 layers whatever the body: deeper slabs, which the update's fit
  // takes for small cells, made the Float64 sum slower (512^3 64-sphere cloud: 3.55 -> 6.37 ms at 16)
  cci::DevTape tape{nullptr, 0, 0, 0};
  double* partial = h->vol_scratch;
  double* res = h->vol_scratch + 2 * cci::calc_volume_blocks();
  cudaError_t e;
  double pd;
  if (h->prec == CC_F64) {
    if ((st = upload_tape<double>(h, body, g->dim, s, &tape)) != CC_OK) return st;
    const cci::DevGrid<double> dg2 = dev_grid<double>(g);
    e = g->dim == 3 ? cci::launch_calc_volume<double, 3>(dg2, tape, partial, res, s)
                    : cci::launch_calc_volume<double, 2>(dg2, tape, partial, res, s);
    pd = dg2.d[0] * dg2.d[1];
    if (g->dim == 3) pd = pd * dg2.d[2];
  } else {
    if ((st = upload_tape<float>(h, body, g->dim, s, &tape)) != CC_OK) return st;
    const cci::DevGrid<float> dg2 = dev_grid<float>(g);
    const bool mx = h->prec == CC_MIXED;
    e = g->dim == 3 ? cci::launch_calc_volume<float, 3>(dg2, tape, partial, res, s, mx)
                    : cci::launch_calc_volume<float, 2>(dg2, tape, partial, res, s, mx);
    float pf = dg2.d[0] * dg2.d[1];
    if (g->dim == 3) pf = pf * dg2.d[2];
    pd = pf;
  }
  if (e != cudaSuccess) return cuda_fail(e, "calc_volume launch");
  double sum = 0.0;
  e = cudaMemcpyAsync(&sum, res, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "calc_volume");
  *out = sum * pd;
  return CC_OK;
}

cc_status cc_monte_carlo_volume(cc_handle* h, const cc_optape* body, const double lo[3], const double hi[3],
                                int64_t n_points, uint64_t seed, int64_t* inside, double* volume, void* stream) {
  if (!h || !lo || !hi || !inside || n_points < 0) return fail(CC_BAD_ARG, "null argument");
  for (int a = 0; a < 3; ++a)
    if (!(hi[a] > lo[a])) return fail(CC_BAD_ARG, "empty box");
  cc_status st = validate_tape(body, 3);
  if (st != CC_OK) return st;
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cci::DevTape tape{nullptr, 0, 0, 0};
  if ((st = upload_tape<double>(h, body, 3, s, &tape)) != CC_OK) return st;
  unsigned long long* cnt = h->rep_scratch;  // the report's counter slots, free between calls
  cudaError_t e = cci::launch_monte_carlo(tape, lo, hi, n_points, seed, cnt, s);
  unsigned long long c = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&c, cnt, sizeof c, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_monte_carlo_volume");
  *inside = (int64_t)c;
  if (volume)
    *volume = n_points > 0 ? double(c) / double(n_points) * ((hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])) : 0.0;
  return CC_OK;
}

cc_status cc_report(cc_handle* h, int64_t ncell, const int8_t* kind, const uint8_t* ambiguous,
                    const void* volume_fraction, int64_t counts[5], double* min_volume_fraction, void* stream) {
  if (!h || !kind || !ambiguous || !volume_fraction || !counts || !min_volume_fraction)
    return fail(CC_BAD_ARG, "null argument");
  if (ncell < 0) return fail(CC_BAD_ARG, "negative cell count");
  DeviceGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  // four counters and the complement of the smallest fraction's bits (0: no cut fraction), zeroed
  // on the device and read back through pinned memory
  unsigned long long res[5] = {0, 0, 0, 0, 0};
  cudaError_t e = cudaSuccess;
  if (ncell > 0) {
    e = cudaMemsetAsync(h->rep_scratch, 0, sizeof res, s);
    if (e == cudaSuccess)
      e = cci::launch_report(ncell, kind, ambiguous, volume_fraction, h->prec == CC_F64, h->rep_scratch,
                             reinterpret_cast<double*>(h->rep_scratch + 4), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->rep_host, h->rep_scratch, sizeof res, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) std::memcpy(res, h->rep_host, sizeof res);
  }
  if (e != cudaSuccess) return cuda_fail(e, "cc_report");
  res[4] = res[4] == 0 ? 0x3FF0000000000000ull : ~res[4];  // no cut cell: 1.0
  counts[0] = ncell;
  counts[1] = (int64_t)res[0];
  counts[2] = (int64_t)res[1];
  counts[3] = (int64_t)res[2];
  counts[4] = (int64_t)res[3];
  std::memcpy(min_volume_fraction, &res[4], sizeof(double));
  return CC_OK;
}

}  // extern "C"
