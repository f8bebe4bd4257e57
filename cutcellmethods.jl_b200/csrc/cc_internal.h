// cc_internal.h -- launch interfaces between the C ABI (capi.cu) and the kernel files.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"

struct cc_handle;

namespace cci {

// Device view of a tiling table blob (include/cutcell_b200.h).
struct DevTable {
  const cc_mc_lut* luts;
  const cc_mc_outcome* outs;
  const cc_mc_tile* tiles;
  const uint8_t* codes;
};

// Where a validated tiling table's parts sit once the blob is at device address `dev`.
struct TableLayout {
  uint32_t n_outcomes = 0, n_tiles = 0;
  DevTable at(const unsigned char* dev) const;
};
// Validate a tiling table blob on the host (every index a kernel reads from it); on failure
// `why` (if not null) receives the reason.
bool check_mc_table(const unsigned char* blob, size_t nbytes, TableLayout* out, std::string* why);

// Grid narrowed to T on the host (convert(CartesianGrid{D,T}, grid)).
template <class T>
struct DevGrid {
  T x0[3];
  T d[3];
  long long n[3];
};

// A tape already in device memory: ops then params (narrowed to T), 8-byte aligned.
struct DevTape {
  const unsigned char* bytes;
  int n_ops;
  int n_params;
  int bytes_len;
  int prunable = 0;  // 1: a union (MIN) of spheres, 2: a smooth union (SMIN) of spheres; see prune_union
  int slab = 8;      // the 3D PLIC passes' pruning slab in cell layers (prune_slab)
};

// The slab depth, in cell layers, over which the 3D PLIC fit and calc_volume prune a union of
// spheres of cell size h: about 0.6 of the median radius, rounded to 4, 8, 16 or 32 layers.
int prune_slab(const cc_optape* t, double h);

struct Cols {
  int8_t* kind;
  uint8_t* amb;
  void* vf;
  void* c;
  void* ff;
  void* fcl;
  void* ic;
};

// Marching cubes: sample (if phi_in == nullptr: sample from the tape into phi_out) and build
// every cell. Returns the CUDA launch status.
// `cut_list` (one slot per cell) and `cut_count` are scratch: the fill pass lists the cut band
// there and the cut pass reads it back.
// With with_cut false only the fill pass runs (the cut band is listed, not built).
template <class T>
cudaError_t launch_mc(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, const DevTable& tb, unsigned* cut_list, unsigned* cut_count,
                      cudaStream_t s, bool with_cut = true, bool mixed = false,
                      void* prune_scratch = nullptr, size_t prune_bytes = 0);
// The mbarrier poll limit of the learned kernels (cc_set_wait_limit): set returns the old value; a
// negative argument restores the default.
long long set_wait_limit(long long polls);
long long wait_limit();
// Scratch launch_mc needs to prune a union-of-spheres tape per fill CTA (n_ops ops per CTA).
size_t mc_prune_bytes(long long n0, long long n1, long long n2, int n_ops, bool f64);
// The handle's pruning scratch, grown to at least `bytes` (null on failure).
void* prune_scratch(cc_handle* h, size_t bytes);

// The learned correction (learned.cu).
int mlp_nparam();
template <class T>
cudaError_t launch_mc_cut_learned(const DevGrid<T>& g, const T* phi, const Cols& cols, const DevTable& tb,
                                  const unsigned* cut_list, const unsigned* cut_count, const float* P, float bound,
                                  unsigned long long* fallback, int* err, cudaStream_t s, bool build);
cudaError_t launch_mlp_grads(const float* P, const float* feats, const float* labels, const float* plain,
                             const float* weights, long long n, unsigned long long seed, int step, int tiles,
                             bool augment, float* grad, float* loss, int* err, cudaStream_t s);
cudaError_t launch_mlp_adam(float* P, float* m, float* v, const float* grad, int tiles, int step, float lr,
                            cudaStream_t s);
cudaError_t launch_mlp_predict(const float* P, const float* feats, long long n, bool correction, float* out, int* err,
                               cudaStream_t s);
cudaError_t launch_labels(const DevGrid<double>& g, const DevTape& tape, const float* phi, const float* vf,
                          const DevTable& tb, const unsigned* list, long long n, float* feats, float* labels,
                          float* plain, int64_t* index, cudaStream_t s);

// `mixed` (Float32 only) selects the FP64 islands of mixed precision; see cc_device.cuh.
template <class T>
cudaError_t launch_ms(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, cudaStream_t s, bool mixed = false);

template <class T>
cudaError_t launch_ms_tree(const T x0[2], const double base_d[2], long long nleaves,
                           const int32_t* level, const int32_t* coord, const DevTape& tape,
                           T* phi4, const Cols& cols, cudaStream_t s, bool mixed = false);

// PLIC update: the fit pass, then the face pass. In 3D the fit records each cell's side (whether
// its plane crosses the cell, or every face is empty or full) in `sides`, one byte per cell, for
// the face pass; 2D takes null.
template <class T, int D>
cudaError_t launch_plic(const DevGrid<T>& g, const DevTape& tape, const Cols& cols, T* normals,
                        T* intercepts, uint8_t* valid, int8_t* sides, cudaStream_t s, bool mixed = false);

// calc_volume partial sums: nblocks (sum, compensation) pairs into `partial`, then a final
// single-block pass into out[0..1]. `partial` holds 2 * calc_volume_blocks() doubles.
int calc_volume_blocks();
// Monte Carlo count of points of the box lo..hi where the body is negative (see plic.cu).
cudaError_t launch_monte_carlo(const DevTape& tape, const double lo[3], const double hi[3], long long npts,
                               unsigned long long seed, unsigned long long* out, cudaStream_t s);
template <class T, int D>
cudaError_t launch_calc_volume(const DevGrid<T>& g, const DevTape& tape, double* partial,
                               double* out, cudaStream_t s, bool mixed = false);

// Op-tape packing (capi.cu): pack a validated host tape for the device (see pack_tape).
template <class T>
size_t pack_tape(const cc_optape* t, int dim, unsigned char* out, int* n_params);
size_t tape_pack_capacity();
int tape_prunable(const cc_optape* t);

// Release the contour a marching-squares handle holds (ms_mesh.cu).
void free_ms_mesh(cc_handle* h);
void free_plic_mesh(cc_handle* h);

// Record the message cc_last_error() returns on this thread.
void set_last_error(const std::string& msg);

// Validate an op-tape for a dim-dimensional grid, and pack + upload it (narrowed to double) into
// the handle's tape buffer on stream s.
cc_status validate_body(const cc_optape* t, int dim);
cc_status upload_body_f64(cc_handle* h, const cc_optape* t, int dim, cudaStream_t s, DevTape* out);
cc_status upload_body_f32(cc_handle* h, const cc_optape* t, int dim, cudaStream_t s, DevTape* out);

cudaError_t launch_report(long long ncell, const int8_t* kind, const uint8_t* amb, const void* vf,
                          int is_f64, unsigned long long* counts, double* vmin, cudaStream_t s);

}  // namespace cci

// The library-side state of one cache (created at allocate_cache time, include/cutcell_b200.h).
namespace cci {
// What a marching-cubes generate_mesh count was taken from, so the emit call that follows can
// start from its block offsets and survivors (mesh.cu).
struct MeshKey {
  bool valid = false;
  uint64_t generation = 0;
  const void* phi = nullptr;
  cc_grid g{};
  int prec = -1;
  unsigned long long tot[3] = {0, 0, 0};
  unsigned long long cut_nodes = 0, cut_cells = 0;  // lengths of the kept survivor lists
};
}  // namespace cci

struct cc_handle {
  int device = 0, method = 0, dim = 3, prec = 0;
  int64_t n[3] = {0, 0, 0};
  bool tree = false;
  unsigned char* tape_dev = nullptr;
  unsigned char* tape_host = nullptr;  // pinned staging
  cudaEvent_t tape_copied = nullptr;
  bool tape_pending = false;
  unsigned char* table_dev = nullptr;
  size_t table_bytes = 0;
  cci::DevTable tb{};
  unsigned* cut_list = nullptr;   // marching cubes: the cut band's cell indices (one slot per cell)
  unsigned* cut_count = nullptr;
  int8_t* plic_sides = nullptr;  // 3D PLIC: the fit's per-cell side bytes for the face pass
  double* vol_scratch = nullptr;  // calc_volume partials + result
  unsigned long long* rep_scratch = nullptr;  // report counters + the complement of the min's bits
  unsigned long long* rep_host = nullptr;     // pinned: the report's results read back
  unsigned* mesh_vbase = nullptr;  // generate_mesh: first vertex of each node's cut edges
  size_t mesh_vbase_n = 0;
  unsigned long long* mesh_scan = nullptr;  // generate_mesh: per-block counts and offsets
  size_t mesh_scan_n = 0;
  unsigned long long* mesh_list = nullptr;  // generate_mesh: cut nodes and cut cells in order
  unsigned long long mesh_node_cap = 0, mesh_cell_cap = 0;
  void* prune = nullptr;  // marching cubes: per fill CTA pruned op lists of a union of spheres
  size_t prune_bytes = 0;
  void* ms_mesh = nullptr;  // marching squares: the last contour built (ms_mesh.cu)
  void* plic_mesh = nullptr;  // PLIC: the last surface count's block offsets (plic_mesh.cu)
  cci::MeshKey mesh_key;      // marching cubes: what the kept mesh count was taken from
  uint64_t generation = 0;    // bumped by every update, so a stored count knows its planes are stale
};

