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

// What each device's table slot holds: the context it was uploaded in (a reset device gets a new
// one, with the array's contents lost) and the blob's size and FNV-1a-64 hash. A call whose table is
// already there skips the upload, so repeated calls copy nothing from the host.
constexpr int kMaxDevices = 64;
struct Resident {
  unsigned long long ctx = 0, hash = 0;
  size_t bytes = 0;
};
Resident g_resident[kMaxDevices];
std::mutex g_scratch_mutex;

typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

// The current context's unique id (0 when the driver cannot say: the table is then re-uploaded).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

unsigned long long fnv1a64(const unsigned char* b, size_t n) {
  unsigned long long h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);  // read back through cc_last_error()
  return s;
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
  const unsigned char* blob = static_cast<const unsigned char*>(table);
  std::string why;
  cci::TableLayout lay;
  if (!cci::check_mc_table(blob, table_bytes, &lay, &why)) return fail(CC_BAD_TABLE, "not a valid tiling table: " + why);

  int old = -1;
  cudaGetDevice(&old);
  if (old != device && cudaSetDevice(device) != cudaSuccess) return fail(CC_CUDA_ERR, "cudaSetDevice failed");
  cc_status status = CC_OK;
  do {
    // The array's device address, looked up on every call with this device current (cheap once
    // the module is loaded; a device reset can move it). In host code the symbol itself is only a
    // host-side stand-in for the array, never its address.
    void* base = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (e != cudaSuccess) {
      status = fail(CC_CUDA_ERR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      break;
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
      std::lock_guard<std::mutex> lk(g_scratch_mutex);
      Resident& r = g_resident[device];
      const unsigned long long ctx = current_context_id();
      const unsigned long long h = fnv1a64(blob, table_bytes);
      if (ctx == 0 || r.ctx != ctx || r.hash != h || r.bytes != table_bytes) {
        r = Resident{};
        e = cudaMemcpyAsync(b, blob, table_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) r = Resident{ctx, h, table_bytes};
      }
    }
    if (e == cudaSuccess) {
      // the launch clears the work list's counter on the stream before the fill pass
      unsigned* count = reinterpret_cast<unsigned*>(b + kCountOffset);
      unsigned* list = reinterpret_cast<unsigned*>(b + kListOffset);
      const cci::DevTable tb = lay.at(b);
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
