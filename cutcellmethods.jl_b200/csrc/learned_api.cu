// learned_api.cu -- C ABI of the learned volume-fraction correction (include/cutcell_b200.h).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_internal.h"

struct cc_mlp {
  int device = 0;
  float* P = nullptr;     // FP32 parameters
  float* m = nullptr;     // Adam first moments
  float* v = nullptr;     // Adam second moments
  float* grad = nullptr;  // per-tile partial gradients [CC_MLP_MAX_TILES][NPARAM]
  float* loss = nullptr;  // per-tile squared-error sums
  int* err = nullptr;     // set by a kernel whose MMA wait ran out
  unsigned long long* fallback = nullptr;
  int step = 0;
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

cc_status check_err(cc_mlp* m, cudaStream_t s) {
  int e = 0;
  cudaError_t c = cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (c == cudaSuccess) c = cudaStreamSynchronize(s);
  if (c != cudaSuccess) return cuda_fail(c, "mlp");
  if (e) {
    cudaMemsetAsync(m->err, 0, sizeof(int), s);
    return fail(CC_DEVICE_TIMEOUT, "a tensor-core MMA did not complete within the wait limit");
  }
  return CC_OK;
}

template <class T>
cci::DevGrid<T> grid_of(const cc_grid* g) {
  cci::DevGrid<T> d;
  for (int a = 0; a < 3; ++a) {
    d.x0[a] = T(g->x0[a]);
    d.d[a] = T(g->d[a]);
    d.n[a] = g->n[a];
  }
  return d;
}

cci::Cols cols_of(const cc_cells* c) {
  return cci::Cols{c->kind, c->ambiguous, c->volume_fraction, c->centroid, c->face_fraction, c->face_centroid_local,
                   c->interface_centroid};
}

bool cells_ok(const cc_cells* c) {
  return c && c->kind && c->ambiguous && c->volume_fraction && c->centroid && c->face_fraction &&
         c->face_centroid_local && c->interface_centroid;
}

cc_status check_mc(cc_handle* h, const cc_grid* g) {
  if (!h || !g) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_MARCHING_CUBES) return fail(CC_BAD_ARG, "handle was created for another method");
  if (g->dim != 3) return fail(CC_DIM_MISMATCH, "grid dimension differs from the cache's");
  for (int a = 0; a < 3; ++a)
    if (g->n[a] != h->n[a]) return fail(CC_DIM_MISMATCH, "grid size differs from the cache's");
  if (!h->table_dev) return fail(CC_NO_TABLE, "no marching-cubes tiling table set on the handle");
  return CC_OK;
}

}  // namespace

extern "C" {

cc_status cc_mlp_create(int32_t device, cc_mlp** out) {
  if (!out) return fail(CC_BAD_ARG, "null argument");
  *out = nullptr;
  if (cci::mlp_nparam() != CC_MLP_NPARAM) return fail(CC_BAD_ARG, "parameter layout mismatch");
  Dev dg(device);
  cc_mlp* m = new cc_mlp();
  m->device = device;
  const size_t pb = CC_MLP_NPARAM * sizeof(float);
  cudaError_t e = cudaMalloc(&m->P, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->m, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->v, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, pb * CC_MLP_MAX_TILES);
  if (e == cudaSuccess) e = cudaMalloc(&m->loss, CC_MLP_MAX_TILES * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&m->fallback, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(m->P, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(m->m, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(m->v, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
  if (e != cudaSuccess) {
    cc_mlp_destroy(m);
    return cuda_fail(e, "cc_mlp_create");
  }
  *out = m;
  return CC_OK;
}

cc_status cc_mlp_destroy(cc_mlp* m) {
  if (!m) return CC_OK;
  Dev dg(m->device);
  cudaFree(m->P);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->grad);
  cudaFree(m->loss);
  cudaFree(m->err);
  cudaFree(m->fallback);
  delete m;
  return CC_OK;
}

cc_status cc_mlp_set_params(cc_mlp* m, const float* params, int32_t n) {
  if (!m || !params || n != CC_MLP_NPARAM) return fail(CC_BAD_ARG, "expected CC_MLP_NPARAM parameters");
  Dev dg(m->device);
  cudaError_t e = cudaMemcpy(m->P, params, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->m, 0, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->v, 0, n * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_set_params");
  m->step = 0;
  return CC_OK;
}

cc_status cc_mlp_get_params(cc_mlp* m, float* params, int32_t n) {
  if (!m || !params || n != CC_MLP_NPARAM) return fail(CC_BAD_ARG, "expected CC_MLP_NPARAM parameters");
  Dev dg(m->device);
  const cudaError_t e = cudaMemcpy(params, m->P, n * sizeof(float), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? CC_OK : cuda_fail(e, "cc_mlp_get_params");
}

cc_status cc_mlp_train(cc_mlp* m, const float* feats, const float* labels, const float* plain,
                       const float* weights, int64_t n, int32_t steps, int32_t tiles, float lr, uint64_t seed,
                       int32_t augment, float* last_loss, void* stream) {
  if (!m || !feats || !labels || n < 1 || steps < 0 || tiles < 1 || tiles > CC_MLP_MAX_TILES)
    return fail(CC_BAD_ARG, "bad training arguments");
  Dev dg(m->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int k = 0; k < steps; ++k) {
    cudaError_t e = cci::launch_mlp_grads(m->P, feats, labels, plain, weights, n, seed, m->step, tiles, augment != 0,
                                          m->grad, m->loss, m->err, s);
    if (e == cudaSuccess) e = cci::launch_mlp_adam(m->P, m->m, m->v, m->grad, tiles, m->step, lr, s);
    if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_train");
    ++m->step;
  }
  cc_status st = check_err(m, s);
  if (st != CC_OK) return st;
  if (last_loss) {
    std::vector<float> l(tiles);
    const cudaError_t e = cudaMemcpy(l.data(), m->loss, tiles * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_train");
    double acc = 0.0;
    for (float x : l) acc += x;
    *last_loss = float(acc / (double(tiles) * 128.0));
  }
  return CC_OK;
}

cc_status cc_mlp_grad(cc_mlp* m, const float* feats, const float* labels, const float* plain, const float* weights,
                      int64_t n, int32_t tiles, uint64_t seed, int32_t step, int32_t augment, float* grad, float* loss,
                      void* stream) {
  if (!m || !feats || !labels || !grad || n < 1 || tiles < 1 || tiles > CC_MLP_MAX_TILES)
    return fail(CC_BAD_ARG, "bad arguments");
  Dev dg(m->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cci::launch_mlp_grads(m->P, feats, labels, plain, weights, n, seed, step, tiles, augment != 0,
                                        m->grad, m->loss, m->err, s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_grad");
  cc_status st = check_err(m, s);
  if (st != CC_OK) return st;
  std::vector<float> g(size_t(tiles) * CC_MLP_NPARAM), l(tiles);
  e = cudaMemcpy(g.data(), m->grad, g.size() * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(l.data(), m->loss, tiles * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_grad");
  for (int i = 0; i < CC_MLP_NPARAM; ++i) {
    float acc = 0.0f;
    for (int b = 0; b < tiles; ++b) acc += g[size_t(b) * CC_MLP_NPARAM + i];
    grad[i] = acc;
  }
  if (loss) {
    double acc = 0.0;
    for (float x : l) acc += x;
    *loss = float(acc / (double(tiles) * 128.0));
  }
  return CC_OK;
}

cc_status cc_mlp_predict(cc_mlp* m, const float* feats, int64_t n, int32_t correction, float* out, void* stream) {
  if (!m || !feats || !out || n < 0) return fail(CC_BAD_ARG, "bad arguments");
  if (n == 0) return CC_OK;
  Dev dg(m->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const cudaError_t e = cci::launch_mlp_predict(m->P, feats, n, correction != 0, out, m->err, s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mlp_predict");
  return check_err(m, s);
}

cc_status cc_mlp_read_weights(const char* path, float* params, int32_t n) {
  if (!path || !params || n != CC_MLP_NPARAM) return fail(CC_BAD_ARG, "expected CC_MLP_NPARAM parameters");
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return fail(CC_BAD_FILE, std::string("cannot open weights file ") + path);
  unsigned char head[64];
  std::vector<unsigned char> body(size_t(n) * 4);
  const bool full = std::fread(head, 1, 64, f) == 64 && std::fread(body.data(), 1, body.size(), f) == body.size();
  const bool at_end = full && std::fgetc(f) == EOF;
  std::fclose(f);
  if (!full || !at_end) return fail(CC_BAD_FILE, "weights file has the wrong length");
  uint32_t version, count;
  float corr, curv;
  uint64_t sum;
  std::memcpy(&version, head + 8, 4);
  std::memcpy(&count, head + 12, 4);
  std::memcpy(&corr, head + 16, 4);
  std::memcpy(&curv, head + 20, 4);
  std::memcpy(&sum, head + 24, 8);
  if (std::memcmp(head, "CCB2MLP1", 8) != 0) return fail(CC_BAD_FILE, "not a weights file (magic)");
  if (version != 1) return fail(CC_BAD_FILE, "unsupported weights file version");
  if (count != uint32_t(CC_MLP_NPARAM)) return fail(CC_BAD_FILE, "weights file holds another network");
  if (corr != CC_MLP_CORRECTION_SCALE || curv != CC_MLP_CURVATURE_NORM)
    return fail(CC_BAD_FILE, "weights file was trained for other correction constants");
  for (int i = 32; i < 64; ++i)
    if (head[i] != 0) return fail(CC_BAD_FILE, "weights file header reserved bytes are not zero");
  uint64_t h = 0xCBF29CE484222325ull;  // FNV-1a 64
  for (unsigned char b : body) {
    h ^= b;
    h *= 0x100000001B3ull;
  }
  if (h != sum) return fail(CC_BAD_FILE, "weights file checksum mismatch");
  std::memcpy(params, body.data(), body.size());  // little-endian host
  return CC_OK;
}

cc_status cc_mc_learned_samples(cc_handle* h, const cc_grid* g, const cc_optape* body, const void* phi,
                                const cc_cells* cells, float* feats, float* labels, float* plain, int64_t* index,
                                int64_t capacity, int64_t* count, void* stream) {
  cc_status st = check_mc(h, g);
  if (st != CC_OK) return st;
  if (h->prec != CC_F32) return fail(CC_BAD_ARG, "training samples are drawn from a Float32 cache");
  if (!phi || !cells_ok(cells) || !feats || !labels || !plain || !count || capacity < 0)
    return fail(CC_BAD_ARG, "null argument");
  if ((st = cci::validate_body(body, 3)) != CC_OK) return st;
  Dev dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned ncut = 0;
  cudaError_t e = cudaMemcpyAsync(&ncut, h->cut_count, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mc_learned_samples");
  const long long n = (long long)ncut < capacity ? (long long)ncut : capacity;
  cci::DevTape tape{nullptr, 0, 0, 0};
  if ((st = cci::upload_body_f64(h, body, 3, s, &tape)) != CC_OK) return st;
  e = cci::launch_labels(grid_of<double>(g), tape, static_cast<const float*>(phi),
                         static_cast<const float*>(cells->volume_fraction), h->tb, h->cut_list, n, feats, labels, plain, index, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mc_learned_samples");
  *count = n;
  return CC_OK;
}

cc_status cc_mc_update_learned(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi,
                               const cc_cells* cells, const cc_mlp* mlp, float bound, int64_t* n_fallback,
                               void* stream) {
  cc_status st = check_mc(h, g);
  if (st != CC_OK) return st;
  if (!mlp || !phi || !cells_ok(cells)) return fail(CC_BAD_ARG, "null argument");
  if (h->prec == CC_MIXED) return fail(CC_BAD_ARG, "the learned correction runs on Float32 or Float64 caches");
  if (!(g->d[0] > 0.0)) return fail(CC_BAD_ARG, "bad grid");
  if ((st = cci::validate_body(body, 3)) != CC_OK) return st;
  Dev dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cc_mlp* m = const_cast<cc_mlp*>(mlp);
  ++h->generation;
  cudaError_t e = cudaMemsetAsync(m->fallback, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "cc_mc_update_learned");
  // The fill and the plain cut-band pass, then the network over the listed cells, reading their
  // plain fractions back. (Building the cells inside the network kernel instead, one fused pass,
  // runs the construction at a third of the plain kernel's occupancy: that kernel's 62 KB of
  // shared memory allow 3 CTAs of 128 threads per SM.)
  constexpr bool split = true;
  if (h->prec == CC_F64) {
    cci::DevTape tape{nullptr, 0, 0, 0};
    if ((st = cci::upload_body_f64(h, body, 3, s, &tape)) != CC_OK) return st;
    const cci::DevGrid<double> dg2 = grid_of<double>(g);
    const size_t pb = tape.prunable ? cci::mc_prune_bytes(g->n[0], g->n[1], g->n[2], tape.n_ops, true) : 0;
    void* ps = pb ? cci::prune_scratch(h, pb) : nullptr;
    e = cci::launch_mc<double>(dg2, tape, nullptr, static_cast<double*>(phi), cols_of(cells), h->tb, h->cut_list,
                               h->cut_count, s, split, false, ps, ps ? pb : 0);
    if (e == cudaSuccess)
      e = cci::launch_mc_cut_learned<double>(dg2, static_cast<const double*>(phi), cols_of(cells), h->tb, h->cut_list,
                                             h->cut_count, m->P, bound, m->fallback, m->err, s, !split);
  } else {
    cci::DevTape tape{nullptr, 0, 0, 0};
    if ((st = cci::upload_body_f32(h, body, 3, s, &tape)) != CC_OK) return st;
    const cci::DevGrid<float> dg2 = grid_of<float>(g);
    const size_t pb = tape.prunable ? cci::mc_prune_bytes(g->n[0], g->n[1], g->n[2], tape.n_ops, false) : 0;
    void* ps = pb ? cci::prune_scratch(h, pb) : nullptr;
    e = cci::launch_mc<float>(dg2, tape, nullptr, static_cast<float*>(phi), cols_of(cells), h->tb, h->cut_list,
                              h->cut_count, s, split, false, ps, ps ? pb : 0);
    if (e == cudaSuccess)
      e = cci::launch_mc_cut_learned<float>(dg2, static_cast<const float*>(phi), cols_of(cells), h->tb, h->cut_list,
                                            h->cut_count, m->P, bound, m->fallback, m->err, s, !split);
  }
  if (e != cudaSuccess) return cuda_fail(e, "cc_mc_update_learned");
  if (n_fallback) {
    unsigned long long fb = 0;
    e = cudaMemcpyAsync(&fb, m->fallback, sizeof fb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "cc_mc_update_learned");
    *n_fallback = (int64_t)fb;
    return check_err(m, s);
  }
  return CC_OK;
}

}  // extern "C"
