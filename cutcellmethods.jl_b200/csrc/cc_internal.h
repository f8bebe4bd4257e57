// cc_internal.h -- launch interfaces between the C ABI (capi.cu) and the kernel files.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"

namespace cci {

// Device view of a tiling table blob (include/cutcell_b200.h).
struct DevTable {
  const cc_mc_lut* luts;
  const cc_mc_outcome* outs;
  const cc_mc_tile* tiles;
  const uint8_t* codes;
};

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
};

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
template <class T>
cudaError_t launch_mc(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, const DevTable& tb, unsigned* cut_list, unsigned* cut_count,
                      cudaStream_t s);

template <class T>
cudaError_t launch_ms(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, cudaStream_t s);

template <class T>
cudaError_t launch_ms_tree(const T x0[2], const double base_d[2], long long nleaves,
                           const int32_t* level, const int32_t* coord, const DevTape& tape,
                           T* phi4, const Cols& cols, cudaStream_t s);

template <class T, int D>
cudaError_t launch_plic(const DevGrid<T>& g, const DevTape& tape, const Cols& cols, T* normals,
                        T* intercepts, uint8_t* valid, cudaStream_t s);

// calc_volume partial sums: nblocks (sum, compensation) pairs into `partial`, then a final
// single-block pass into out[0..1]. `partial` holds 2 * calc_volume_blocks() doubles.
int calc_volume_blocks();
template <class T, int D>
cudaError_t launch_calc_volume(const DevGrid<T>& g, const DevTape& tape, double* partial,
                               double* out, cudaStream_t s);

// Record the message cc_last_error() returns on this thread.
void set_last_error(const std::string& msg);

cudaError_t launch_report(long long ncell, const int8_t* kind, const uint8_t* amb, const void* vf,
                          int is_f64, unsigned long long* counts, double* vmin, cudaStream_t s);

}  // namespace cci
