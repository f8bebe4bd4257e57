// noalloc.cu -- marching cubes from a given nodal field, for callers that cannot allocate.
//
// Some callers may not let a library allocate device memory: a solver whose device memory is
// carved out of its own pool up front and budgeted to the byte, or a time-stepping loop where a
// cudaMalloc (which can synchronize the whole device) in the middle of a step is not acceptable.
// cc_mc_cells_from_phi_noalloc serves them. The caller passes the nodal field and the output
// columns, as for cc_mc_cells_from_phi; the only scratch the marching-cubes passes need -- the
// tiling table's device copy and the cut-band work list -- lives in one file-scope device array
// below, which every GPU that loads this library holds until the process exits. Nothing here
// calls cudaMalloc, cudaFree or any allocating library routine.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_internal.h"

namespace {

// Largest grid the static work list can serve: 2^23 cells (for example 203^3, or 512 x 128 x 128).
constexpr long long kMaxCells = 8388608;
constexpr size_t kTableBytes = 64 * 1024;    // the tiling table's device copy
constexpr size_t kCountOffset = kTableBytes;  // the work list's counter
constexpr size_t kListOffset = kTableBytes + 256;
constexpr size_t kScratchBytes = kListOffset + size_t(kMaxCells) * sizeof(unsigned);  // 32 MiB + 64.25 KiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's device address per device, looked up once with that device current. In host code
// the symbol g_noalloc_scratch is only a host-side stand-in for the array, never its address.
constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);  // read back through cc_last_error()
  return s;
}

bool table_ok(const unsigned char* b, size_t nbytes, cci::DevTable* tb, unsigned char* dev_base) {
  if (nbytes < sizeof(cc_mc_table_header) + 256 * sizeof(cc_mc_lut)) return false;
  cc_mc_table_header hd;
  std::memcpy(&hd, b, sizeof hd);
  if (hd.magic != CC_MC_TABLE_MAGIC || hd.version != 1 || hd.total_bytes != nbytes) return false;
  const size_t need = sizeof hd + 256 * sizeof(cc_mc_lut) + hd.n_outcomes * sizeof(cc_mc_outcome) +
                      hd.n_tiles * sizeof(cc_mc_tile) + hd.n_codes;
  if (need > nbytes || hd.n_outcomes > 65535 || hd.n_tiles > 65535) return false;
  const cc_mc_lut* luts = reinterpret_cast<const cc_mc_lut*>(b + sizeof hd);
  const cc_mc_outcome* outs = reinterpret_cast<const cc_mc_outcome*>(luts + 256);
  const cc_mc_tile* tiles = reinterpret_cast<const cc_mc_tile*>(outs + hd.n_outcomes);
  const uint8_t* codes = reinterpret_cast<const uint8_t*>(tiles + hd.n_tiles);
  for (int l = 0; l < 256; ++l) {
    const cc_mc_lut& e = luts[l];
    if (e.ntests > 6 || e.lcase < 1 || e.lcase > 15) return false;
    if (size_t(e.outcome_base) + (size_t(1) << e.ntests) > hd.n_outcomes) return false;
    for (int i = 0; i < e.ntests; ++i)
      if (e.face[i] == 0 || e.face[i] > 6 || e.face[i] < -6) return false;
  }
  for (uint32_t o = 0; o < hd.n_outcomes; ++o)
    if (outs[o].itype > CC_MC_INTERIOR_EDGE || outs[o].edge > 11 || outs[o].tile_true >= hd.n_tiles ||
        outs[o].tile_false >= hd.n_tiles)
      return false;
  for (uint32_t t = 0; t < hd.n_tiles; ++t) {
    if (tiles[t].ntris > 16 || size_t(tiles[t].code_off) + 3u * tiles[t].ntris > hd.n_codes) return false;
    for (int c = 0; c < 3 * tiles[t].ntris; ++c)
      if (codes[tiles[t].code_off + c] < 1 || codes[tiles[t].code_off + c] > 13) return false;
  }
  tb->luts = reinterpret_cast<const cc_mc_lut*>(dev_base + sizeof hd);
  tb->outs = reinterpret_cast<const cc_mc_outcome*>(tb->luts + 256);
  tb->tiles = reinterpret_cast<const cc_mc_tile*>(tb->outs + hd.n_outcomes);
  tb->codes = reinterpret_cast<const uint8_t*>(tb->tiles + hd.n_tiles);
  return true;
}

}  // namespace

extern "C" cc_status cc_mc_cells_from_phi_noalloc(int32_t device, int32_t prec, const cc_grid* g,
                                                  const void* table, size_t table_bytes, const void* phi,
                                                  const cc_cells* cells, void* stream) {
  if (!g || !table || !phi || !cells || !cells->kind || !cells->ambiguous || !cells->volume_fraction ||
      !cells->centroid || !cells->face_fraction || !cells->face_centroid_local || !cells->interface_centroid)
    return fail(CC_BAD_ARG, "null argument");
  if (device < 0 || device >= kMaxDevices) return fail(CC_BAD_ARG, "device index out of range");
  if (prec != CC_F32 && prec != CC_F64) return fail(CC_BAD_ARG, "unsupported precision");
  if (g->dim != 3) return fail(CC_BAD_ARG, "marching cubes needs a 3D grid");
  for (int a = 0; a < 3; ++a)
    if (g->n[a] < 1 || !(g->d[a] > 0.0)) return fail(CC_BAD_ARG, "bad grid");
  const double ncell = double(g->n[0]) * double(g->n[1]) * double(g->n[2]);
  if (ncell > double(kMaxCells)) {
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "grid has %.0f cells; the allocation-free entry point serves at most %lld cells (its work "
                  "list is a fixed device array) -- use cc_mc_cells_from_phi with a handle instead",
                  ncell, kMaxCells);
    return fail(CC_TOO_LARGE, buf);
  }
  if (table_bytes > kTableBytes) return fail(CC_BAD_TABLE, "tiling table larger than the 64 KiB table slot");

  int old = -1;
  cudaGetDevice(&old);
  if (old != device && cudaSetDevice(device) != cudaSuccess) return fail(CC_CUDA_ERR, "cudaSetDevice failed");
  cc_status status = CC_OK;
  do {
    void* base = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_scratch_mutex);
      if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
          status = fail(CC_CUDA_ERR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
          break;
        }
        g_scratch_addr[device] = p;
      }
      base = g_scratch_addr[device];
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    cci::DevTable tb{};
    if (!table_ok(static_cast<const unsigned char*>(table), table_bytes, &tb, b)) {
      status = fail(CC_BAD_TABLE, "not a valid tiling table");
      break;
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(b, table, table_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      // the launch clears the work list's counter on the stream before the fill pass
      unsigned* count = reinterpret_cast<unsigned*>(b + kCountOffset);
      unsigned* list = reinterpret_cast<unsigned*>(b + kListOffset);
      cci::Cols cols{cells->kind, cells->ambiguous, cells->volume_fraction, cells->centroid, cells->face_fraction,
                     cells->face_centroid_local, cells->interface_centroid};
      cci::DevTape none{nullptr, 0, 0, 0};
      if (prec == CC_F64) {
        cci::DevGrid<double> dg;
        for (int a = 0; a < 3; ++a) { dg.x0[a] = g->x0[a]; dg.d[a] = g->d[a]; dg.n[a] = g->n[a]; }
        e = cci::launch_mc<double>(dg, none, static_cast<const double*>(phi), nullptr, cols, tb, list, count, s);
      } else {
        cci::DevGrid<float> dg;
        for (int a = 0; a < 3; ++a) { dg.x0[a] = float(g->x0[a]); dg.d[a] = float(g->d[a]); dg.n[a] = g->n[a]; }
        e = cci::launch_mc<float>(dg, none, static_cast<const float*>(phi), nullptr, cols, tb, list, count, s);
      }
    }
    if (e != cudaSuccess) status = fail(CC_CUDA_ERR, std::string("marching cubes launch: ") + cudaGetErrorString(e));
  } while (false);
  if (old >= 0 && old != device) cudaSetDevice(old);
  return status;
}
