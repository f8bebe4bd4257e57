// learned.cu -- the learned volume-fraction correction on sm_100a tensor cores (tcgen05).
//
// A small MLP, 8 -> 64 -> 64 -> 1 with GELU hidden layers and a sigmoid output p, corrects the
// fluid volume fraction that marching cubes gives a cut cell from the cell's corner values scaled
// by the cell size (x = phi / h, marching-cubes corner order). It is trained on the fluid
// fractions that marching cubes gives the same cells at 8x sub-refinement. Only a cut cell's
// volume_fraction is replaced; kind and the face fractions stay the plain construction's, so
// watertightness and the shared-face identities survive. Where the correction is not finite,
// exceeds `bound` or takes the value out of [0, 1], the plain value is kept.
//
// The correction is first order in the curvature. Marching cubes is exact for a planar
// interface, and its volume error on a curved one is about h / R. In the corner values the
// curvature shows only as the four non-linear Walsh components q (the xy, xz, yz and xyz
// patterns of the 8 corners), of size about h / R. Scale-free features cannot tell a fine
// grid's small correction from a coarse grid's large one, so a network fed x directly, trained on
// coarse grids, over-corrects fine ones. So the network sees x with its non-linear part rescaled
// to a fixed norm K0,
//     x~ = lin(x) + quad(x) K0 / |quad(x)|,      s = |quad(x)| / K0,
// and the correction is homogeneous of degree one in the curvature:
//     corrected = plain + s * CORR * (2 p(x~) - 1),      CORR = CC_MLP_CORRECTION_SCALE.
// A planar cell (quad = 0) is left as it is.
//
// Every GEMM runs on the 5th-generation tensor cores: BF16 operands staged in shared memory in the
// K-major "interleaved" layout (8-row x 16-byte core matrices), FP32 accumulators in tensor memory
// (TMEM), one tcgen05.mma per K = 16 step issued by one thread, completion signalled through an
// mbarrier by tcgen05.commit, results read back with tcgen05.ld (warp w reads TMEM lanes 32w..).
// A CTA works on tiles of 128 samples (the MMA's M): row t of every activation tile is sample t,
// which thread t owns.
//
// Precision. The curvature of the interface shows in the corner values only as second
// differences of order (h / R) -- a few 1e-3 of the values themselves on fine grids, below one
// BF16 rounding step. So the forward GEMMs run split: every operand v is a BF16 pair
// hi = bf16(v), lo = bf16(v - hi), and a product is hi*hi + lo*hi + hi*lo (three MMAs into the
// same FP32 accumulator), about 16 significant bits. The backward GEMMs use the high parts only
// (a gradient needs no such precision).
//
//   forward   H1 = X W1^T (K 16, x3)     A1 = gelu(H1 + b1)
//             H2 = A1 W2^T (K 64, x3)    z = gelu(H2 + b2) . w3 + b3,  p = sigmoid(z)
//   backward  dW2 = dH2^T A1 (K = 128 samples),  dA1 = dH2 W2 (K 64),  dW1 = dH1^T X (K = 128)
//
// Training minimises the mean over a step's samples of w |c - (label - plain)| (c the correction
// above, w a per-sample weight), or, without plain fractions, the mean squared error of p
// against the labels (the network alone). It writes per-CTA partial gradients to fixed slots and
// a second kernel sums them in CTA order and takes an Adam step, so training is deterministic.
#include <cstdint>
#include <cstring>
#include <cuda_bf16.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"
#include "mc_cell.cuh"

namespace {

using namespace ccd;
using namespace ccmc;
using cci::Cols;
using cci::DevGrid;
using cci::DevTape;

constexpr int TILE = 128;  // samples per tile = MMA M = threads per CTA
constexpr int H = 64;      // hidden width
constexpr int KIN = 16;    // 8 inputs padded to one K step
constexpr float CORR = CC_MLP_CORRECTION_SCALE;
constexpr float K0 = CC_MLP_CURVATURE_NORM;

// FP32 parameter vector layout
constexpr int P_W1 = 0;            // [64][8]  (row = output unit)
constexpr int P_B1 = P_W1 + 64 * 8;
constexpr int P_W2 = P_B1 + 64;    // [64][64]
constexpr int P_B2 = P_W2 + 64 * 64;
constexpr int P_W3 = P_B2 + 64;    // [64]
constexpr int P_B3 = P_W3 + 64;
constexpr int NPARAM = P_B3 + 1;   // 4801
static_assert(NPARAM == CC_MLP_NPARAM, "parameter layout");

constexpr long long WAIT_LIMIT = 1ll << 22;  // default mbarrier polls before a tile gives up

// ---------------------------------------------------------------------------------------------
// tcgen05 / mbarrier primitives
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle. lbo = bytes between core matrices
// adjacent along K, sbo = bytes between core matrices adjacent along M (or N).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version 1 (sm_100)
  return d;                // base offset 0, layout type 0 = no swizzle
}
// Instruction descriptor, kind::f16: BF16 A and B, FP32 accumulator, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an MMA commit: false after `limit` polls or about one second (the clock starts
// after 256 polls).
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity, long long limit) {
  unsigned long long t0 = 0;
  for (long long i = 0; i < limit; ++i) {
    if (mbar_try_wait(m, parity)) return true;
    if ((i & 255) == 255) {
      if (t0 == 0) t0 = global_ns();
      else if (global_ns() - t0 > 1000000000ull) return false;
    }
  }
  return false;
}
// 16 consecutive FP32 accumulator columns of this thread's TMEM lane, waited for before use.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of bf16 element (r, k) of an [R x K] tile stored K-major as 8x8 core matrices:
// core (r/8, k/8) at ((r/8)(K/8) + k/8) * 128 bytes, element at (r%8)*16 + (k%8)*2 within it.
__device__ __forceinline__ int kmaj(int r, int k, int K) {
  return ((((r >> 3) * (K >> 3)) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1);
}
__device__ __forceinline__ unsigned short bf16_bits(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
__device__ __forceinline__ float bf16_val(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
// v = hi + lo to about 16 significant bits, both BF16
__device__ __forceinline__ void split_bf16(float v, unsigned short& hi, unsigned short& lo) {
  hi = bf16_bits(v);
  lo = bf16_bits(v - bf16_val(hi));
}
__device__ __forceinline__ void put_bits(unsigned char* tile, int r, int k, int K, unsigned short b) {
  *reinterpret_cast<unsigned short*>(tile + kmaj(r, k, K)) = b;
}
__device__ __forceinline__ void put_bf16(unsigned char* tile, int r, int k, int K, float v) {
  put_bits(tile, r, k, K, bf16_bits(v));
}
// Row r, columns k0..k0+7 (k0 a multiple of 8): one 16-byte store.
__device__ __forceinline__ void put_row8(unsigned char* tile, int r, int k0, int K, const unsigned short (&b)[8]) {
  uint4 w;
  w.x = (uint32_t)b[0] | ((uint32_t)b[1] << 16);
  w.y = (uint32_t)b[2] | ((uint32_t)b[3] << 16);
  w.z = (uint32_t)b[4] | ((uint32_t)b[5] << 16);
  w.w = (uint32_t)b[6] | ((uint32_t)b[7] << 16);
  *reinterpret_cast<uint4*>(tile + kmaj(r, k0, K)) = w;
}
// D[M x N] (+)= A[M x K] B[N x K]^T over K / 16 MMAs; tiles in the layout above. With acc false
// the first MMA overwrites D.
__device__ __forceinline__ void gemm_kmaj(uint32_t tmem_d, const unsigned char* A, const unsigned char* B, int M,
                                          int N, int K, bool acc) {
  const uint32_t idesc = umma_idesc(M, N);
  const uint32_t sbo = (uint32_t)(K / 8) * 128u;
  for (int s = 0; s < K / 16; ++s) {
    const uint64_t da = umma_desc(smem_u32(A) + 256u * s, 128u, sbo);
    const uint64_t db = umma_desc(smem_u32(B) + 256u * s, 128u, sbo);
    umma_bf16(tmem_d, da, db, idesc, (acc || s > 0) ? 1u : 0u);
  }
}
// D = A B^T in split precision: Ah Bh + Al Bh + Ah Bl.
__device__ __forceinline__ void gemm_split(uint32_t tmem_d, const unsigned char* Ah, const unsigned char* Al,
                                           const unsigned char* Bh, const unsigned char* Bl, int M, int N, int K) {
  gemm_kmaj(tmem_d, Ah, Bh, M, N, K, false);
  gemm_kmaj(tmem_d, Al, Bh, M, N, K, true);
  gemm_kmaj(tmem_d, Ah, Bl, M, N, K, true);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Shared-memory layout (bytes) of an MLP CTA.
struct MlpLayout {
  static constexpr int XH = 0;                          // [128 x 16] inputs, high parts
  static constexpr int XL = XH + TILE * KIN * 2;        // low parts
  static constexpr int W1H = XL + TILE * KIN * 2;       // [64 x 16]
  static constexpr int W1L = W1H + H * KIN * 2;
  static constexpr int A1H = W1L + H * KIN * 2;         // [128 x 64]
  static constexpr int A1L = A1H + TILE * H * 2;
  static constexpr int W2H = A1L + TILE * H * 2;        // [64 x 64]
  static constexpr int W2L = W2H + H * H * 2;
  static constexpr int INFER_BYTES = W2L + H * H * 2;   // all that inference reads
  static constexpr int W2T = INFER_BYTES;               // [64 x 64] W2^T, high parts (training)
  static constexpr int DH2 = W2T + H * H * 2;           // [128 x 64]
  static constexpr int DH2T = DH2 + TILE * H * 2;       // [128 x 128], rows 64.. zero
  static constexpr int A1T = DH2T + TILE * TILE * 2;    // [64 x 128], high parts
  static constexpr int DH1T = A1T + H * TILE * 2;       // [128 x 128], rows 64.. zero
  static constexpr int XT = DH1T + TILE * TILE * 2;     // [16 x 128]: rows 0..7 high, 8..15 low parts
  static constexpr int H1 = XT + KIN * TILE * 2;        // f32 [128][65]
  static constexpr int TRAIN_PAR = H1 + TILE * 65 * 4;
  static constexpr int PAR_FLOATS = 3 * H + 8;          // b1[64] b2[64] w3[64] b3, then 4 scratch
  static constexpr int RED_FLOATS = 4 * 3 * H;          // per-warp partial sums of db1, db2, dw3
  static constexpr int INFER_SMEM = INFER_BYTES + PAR_FLOATS * 4 + 64;
  static constexpr int TRAIN_BYTES = TRAIN_PAR + (PAR_FLOATS + RED_FLOATS) * 4 + 64;
};
static_assert(MlpLayout::TRAIN_BYTES <= 227 * 1024, "training CTA exceeds shared memory");

struct MlpShared {
  unsigned char* base;
  float* par;
  float* red;  // training only
  uint64_t* mbar;
  uint32_t* tmem;
  long long limit;  // mbarrier polls before an MMA wait gives up (cc_set_wait_limit)
};

__device__ __forceinline__ MlpShared mlp_shared(unsigned char* smem, bool train, long long limit) {
  MlpShared s;
  s.base = smem;
  s.limit = limit;
  const int par = train ? MlpLayout::TRAIN_PAR : MlpLayout::INFER_BYTES;
  s.par = reinterpret_cast<float*>(smem + par);
  s.red = s.par + MlpLayout::PAR_FLOATS;
  const int misc = par + (MlpLayout::PAR_FLOATS + (train ? MlpLayout::RED_FLOATS : 0)) * 4;
  s.mbar = reinterpret_cast<uint64_t*>(smem + ((misc + 7) / 8) * 8);
  s.tmem = reinterpret_cast<uint32_t*>(s.mbar + 1);
  return s;
}

// Stage the weights (FP32 master copy -> BF16 high/low tiles) and biases of the network.
__device__ void stage_weights(const float* __restrict__ P, const MlpShared& s, bool train) {
  unsigned char* b = s.base;
  for (int e = threadIdx.x; e < H * KIN; e += TILE) {
    const int j = e / KIN, k = e % KIN;
    unsigned short hi, lo;
    split_bf16(k < 8 ? P[P_W1 + j * 8 + k] : 0.0f, hi, lo);
    put_bits(b + MlpLayout::W1H, j, k, KIN, hi);
    put_bits(b + MlpLayout::W1L, j, k, KIN, lo);
  }
  for (int e = threadIdx.x; e < H * H; e += TILE) {
    const int j = e / H, i = e % H;
    unsigned short hi, lo;
    split_bf16(P[P_W2 + j * H + i], hi, lo);
    put_bits(b + MlpLayout::W2H, j, i, H, hi);
    put_bits(b + MlpLayout::W2L, j, i, H, lo);
    if (train) put_bits(b + MlpLayout::W2T, i, j, H, hi);
  }
  // par: b1[64], b2[64], w3[64], b3
  for (int e = threadIdx.x; e < 3 * H + 1; e += TILE)
    s.par[e] = e < H ? P[P_B1 + e] : e < 2 * H ? P[P_B2 + e - H] : e < 3 * H ? P[P_W3 + e - 2 * H] : P[P_B3];
}

// Wait for the MMAs committed to the CTA's mbarrier; false on every thread if any thread's wait
// ran out.
// Before the caller gives up (and frees the TMEM the MMAs write), thread 0 waits once more, with
// the default limit, for the MMAs already committed, so none is still in flight when the CTA
// releases its TMEM.
__device__ __forceinline__ bool mma_done(const MlpShared& s, uint32_t& phase) {
  const bool ok = mbar_wait(s.mbar, phase, s.limit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) mbar_wait(s.mbar, phase, WAIT_LIMIT);
    __syncthreads();
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

// One tile's forward pass. x: this thread's 8 inputs (zeros for a padding row). In training,
// keeps what the backward pass needs in shared memory and the H2 accumulator in TMEM columns
// 0..63. `phase` is the running mbarrier parity. Returns false if an MMA never completed.
__device__ bool mlp_forward(const MlpShared& s, uint32_t tmem, const float x[8], bool train, uint32_t& phase,
                            float& z_out) {
  unsigned char* b = s.base;
  const int t = threadIdx.x;
  {
    unsigned short hi[8], lo[8];
    const unsigned short zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; ++k) split_bf16(x[k], hi[k], lo[k]);
    put_row8(b + MlpLayout::XH, t, 0, KIN, hi);
    put_row8(b + MlpLayout::XH, t, 8, KIN, zero);
    put_row8(b + MlpLayout::XL, t, 0, KIN, lo);
    put_row8(b + MlpLayout::XL, t, 8, KIN, zero);
    if (train) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        put_bits(b + MlpLayout::XT, k, t, TILE, hi[k]);
        put_bits(b + MlpLayout::XT, 8 + k, t, TILE, lo[k]);
      }
    }
  }
  fence_async_smem();
  __syncthreads();
  if (t == 0) {
    tc_fence_after();
    gemm_split(tmem, b + MlpLayout::XH, b + MlpLayout::XL, b + MlpLayout::W1H, b + MlpLayout::W1L, TILE, H, KIN);
    umma_commit(s.mbar);
  }
  if (!mma_done(s, phase)) return false;
  const uint32_t lane_addr = tmem + ((uint32_t)(32 * (t / 32)) << 16);
  float* h1row = reinterpret_cast<float*>(b + MlpLayout::H1) + t * 65;
  for (int c = 0; c < H / 16; ++c) {
    float v[16];
    tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      unsigned short hi[8], lo[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = 16 * c + 8 * half + q;
        const float h = v[8 * half + q] + s.par[j];
        split_bf16(gelu(h), hi[q], lo[q]);
        if (train) {
          h1row[j] = h;
          put_bits(b + MlpLayout::A1T, j, t, TILE, hi[q]);
        }
      }
      put_row8(b + MlpLayout::A1H, t, 16 * c + 8 * half, H, hi);
      put_row8(b + MlpLayout::A1L, t, 16 * c + 8 * half, H, lo);
    }
  }
  tc_fence_before();
  fence_async_smem();
  __syncthreads();
  if (t == 0) {
    tc_fence_after();
    gemm_split(tmem, b + MlpLayout::A1H, b + MlpLayout::A1L, b + MlpLayout::W2H, b + MlpLayout::W2L, TILE, H, H);
    umma_commit(s.mbar);
  }
  if (!mma_done(s, phase)) return false;
  float z = 0.0f;
  for (int c = 0; c < H / 16; ++c) {
    float v[16];
    tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int j = 16 * c + q;
      z = z + gelu(v[q] + s.par[H + j]) * s.par[2 * H + j];
    }
  }
  z_out = z + s.par[3 * H];
  return true;
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sum over the 128 threads of the CTA, in a fixed order; every thread gets the result.
__device__ __forceinline__ float cta_sum(float v, float* red4) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red4[threadIdx.x / 32] = v;
  __syncthreads();
  const float r = (red4[0] + red4[1]) + (red4[2] + red4[3]);
  __syncthreads();
  return r;
}

// The image of marching-cubes corner c under cube symmetry `sym` (0..47): the axes permuted by
// sym % 6, then reflected along the axes whose bit is set in sym / 6. Corner bits in
// marching-cubes order: c0 (0,0,0) c1 (1,0,0) c2 (1,1,0) c3 (0,1,0), c4..c7 the same at z = 1.
__device__ __forceinline__ int sym_corner(int c, unsigned sym) {
  const int b[3] = {((c & 3) == 1 || (c & 3) == 2) ? 1 : 0, (c & 3) >= 2 ? 1 : 0, c >= 4 ? 1 : 0};
  const unsigned char perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  const unsigned pi = sym % 6u, f = sym / 6u;
  int o[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) o[a] = b[perm[pi][a]] ^ (int)((f >> a) & 1u);
  return 4 * o[2] + (o[1] ? (o[0] ? 2 : 3) : (o[0] ? 1 : 0));
}

// The network input of a cell, x~ = lin(x) + quad(x) K0 / |quad(x)|, and the scale s = |quad(x)| /
// K0 of its correction (0 for a cell whose corner values are exactly trilinear-free, which keeps
// x). quad(x) is the projection of x on the corner patterns sx*sy, sx*sz, sy*sz and sx*sy*sz
// (s = -1 / +1 per corner bit), which are orthogonal to the constant and linear ones.
__device__ __forceinline__ void homogenize(const float x[8], float xt[8], float& s) {
  const float sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const float sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const float sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  float qxy = 0.0f, qxz = 0.0f, qyz = 0.0f, qxyz = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    qxy += sx[c] * sy[c] * x[c];
    qxz += sx[c] * sz[c] * x[c];
    qyz += sy[c] * sz[c] * x[c];
    qxyz += sx[c] * sy[c] * sz[c] * x[c];
  }
  qxy *= 0.125f; qxz *= 0.125f; qyz *= 0.125f; qxyz *= 0.125f;
  float quad[8], nn = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    quad[c] = qxy * (sx[c] * sy[c]) + qxz * (sx[c] * sz[c]) + qyz * (sy[c] * sz[c]) + qxyz * (sx[c] * sy[c] * sz[c]);
    nn += quad[c] * quad[c];
  }
  const float qn = sqrtf(nn);
  if (!(qn > 0.0f)) {
#pragma unroll
    for (int c = 0; c < 8; ++c) xt[c] = x[c];
    s = 0.0f;
    return;
  }
  const float f = K0 / qn - 1.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) xt[c] = x[c] + quad[c] * f;
  s = qn / K0;
}

// ---------------------------------------------------------------------------------------------
// Training: one tile of 128 samples per CTA per step; per-CTA partial gradients in grad[cta][].
__global__ void __launch_bounds__(TILE, 1)
    mlp_train_kernel(const float* __restrict__ P, const float* __restrict__ feats, const float* __restrict__ labels,
                     const float* __restrict__ plain, const float* __restrict__ weights, long long n,
                     unsigned long long seed, int step, int augment, float inv_batch, float* __restrict__ grad,
                     float* __restrict__ loss, int* __restrict__ err, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem[];
  const MlpShared s = mlp_shared(smem, true, wait_limit);
  const int t = threadIdx.x, warp = t / 32, lane = t & 31;
  unsigned char* b = s.base;
  stage_weights(P, s, true);
  // rows 64..127 of the transposed gradient tiles stay zero (M is padded to 128)
  for (int e = t; e < TILE * TILE / 2; e += TILE) {
    const int r = 64 + e / TILE, k = e % TILE;
    put_bits(b + MlpLayout::DH2T, r, k, TILE, 0);
    put_bits(b + MlpLayout::DH1T, r, k, TILE, 0);
  }
  if (t == 0) mbar_init(s.mbar, 1);
  if (t < 32) { tmem_alloc(s.tmem, 128); tmem_relinquish(); }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem;
  uint32_t phase = 0;
  float* red4 = s.par + 3 * H + 4;  // 4 floats of scratch past b3
  float* g = grad + (long long)blockIdx.x * NPARAM;

  // the sample: a counter-based hash of (seed, step, slot), uniform over the data set; its high
  // bits pick the cube symmetry applied to it
  unsigned long long hsh = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(step * (long long)gridDim.x * TILE +
                                                                                  blockIdx.x * TILE + t + 1));
  hsh ^= hsh >> 33; hsh *= 0xff51afd7ed558ccdull; hsh ^= hsh >> 33; hsh *= 0xc4ceb9fe1a85ec53ull; hsh ^= hsh >> 33;
  const long long idx = (long long)(hsh % (unsigned long long)n);
  const unsigned sym = augment ? (unsigned)((hsh >> 40) % 48ull) : 0u;
  float xr[8], x[8], sc = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) xr[sym_corner(k, sym)] = feats[idx * 8 + k];
  const bool corr_mode = plain != nullptr;
  if (corr_mode) homogenize(xr, x, sc);
  else {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = xr[k];
  }
  // the target: p itself, or the correction that turns the plain fraction into the label
  const float y = corr_mode ? labels[idx] - plain[idx] : labels[idx];
  const float w = weights ? weights[idx] : 1.0f;

  bool ok = true;
  float z = 0.0f;
  do {
    if (!mlp_forward(s, tmem, x, true, phase, z)) { ok = false; break; }
    const float p = sigmoidf_(z);
    float l, dz;
    if (corr_mode) {  // w |c - y|, c = s CORR (2p - 1)
      const float e = sc * CORR * (2.0f * p - 1.0f) - y;
      const float sg = e > 0.0f ? 1.0f : (e < 0.0f ? -1.0f : 0.0f);
      l = w * fabsf(e);
      dz = inv_batch * w * sg * sc * (2.0f * CORR) * p * (1.0f - p);
    } else {          // w (p - y)^2
      const float e = p - y;
      l = w * e * e;
      dz = 2.0f * e * inv_batch * w * p * (1.0f - p);
    }
    l = cta_sum(l, red4);
    if (t == 0) loss[blockIdx.x] = l;
    const float db3 = cta_sum(dz, red4);
    if (t == 0) g[P_B3] = db3;
    // layer 3 and the gradient into H2, from the still-resident H2 accumulator in TMEM
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    for (int c = 0; c < H / 16; ++c) {
      float v[16];
      tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        unsigned short d16[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int j = 16 * c + 8 * half + q;
          const float h2 = v[8 * half + q] + s.par[H + j];
          const float a2 = gelu(h2);
          const float dw3 = warp_sum(dz * a2);
          const float dh2 = dz * s.par[2 * H + j] * gelu_grad(h2);
          const float db2 = warp_sum(dh2);
          if (lane == 0) {
            s.red[(warp * 3 + 2) * H + j] = dw3;
            s.red[(warp * 3 + 1) * H + j] = db2;
          }
          d16[q] = bf16_bits(dh2);
          put_bits(b + MlpLayout::DH2T, j, t, TILE, d16[q]);
        }
        put_row8(b + MlpLayout::DH2, t, 16 * c + 8 * half, H, d16);
      }
    }
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      gemm_kmaj(tmem, b + MlpLayout::DH2T, b + MlpLayout::A1T, TILE, H, TILE, false);   // dW2 -> cols 0..63
      gemm_kmaj(tmem + H, b + MlpLayout::DH2, b + MlpLayout::W2T, TILE, H, H, false);   // dA1 -> cols 64..127
      umma_commit(s.mbar);
    }
    if (!mma_done(s, phase)) { ok = false; break; }
    const float* h1row = reinterpret_cast<const float*>(b + MlpLayout::H1) + t * 65;
    for (int c = 0; c < H / 16; ++c) {
      float v[16];
      tmem_ld16(lane_addr + H + 16 * c, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int i = 16 * c + q;
        const float dh1 = v[q] * gelu_grad(h1row[i]);
        const float db1 = warp_sum(dh1);
        if (lane == 0) s.red[(warp * 3 + 0) * H + i] = db1;
        put_bf16(b + MlpLayout::DH1T, i, t, TILE, dh1);
      }
    }
    if (t < 64) {  // TMEM lanes 0..63 hold dW2's rows (output units)
      for (int c = 0; c < H / 16; ++c) {
        float v[16];
        tmem_ld16(lane_addr + 16 * c, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) g[P_W2 + t * H + 16 * c + q] = v[q];
      }
    }
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      gemm_kmaj(tmem, b + MlpLayout::DH1T, b + MlpLayout::XT, TILE, KIN, TILE, false);  // dW1 -> cols 0..15
      umma_commit(s.mbar);
    }
    if (!mma_done(s, phase)) { ok = false; break; }
    if (t < 64) {
      float v[16];
      tmem_ld16(lane_addr, v);
#pragma unroll
      for (int k = 0; k < 8; ++k) g[P_W1 + t * 8 + k] = v[k] + v[8 + k];  // high + low parts of x
      // the bias and output-weight gradients: the four warps' partial sums, in warp order
      const float* r = s.red;
      g[P_B1 + t] = (r[0 * H + t] + r[3 * H + t]) + (r[6 * H + t] + r[9 * H + t]);
      g[P_B2 + t] = (r[1 * H + t] + r[4 * H + t]) + (r[7 * H + t] + r[10 * H + t]);
      g[P_W3 + t] = (r[2 * H + t] + r[5 * H + t]) + (r[8 * H + t] + r[11 * H + t]);
    }
  } while (false);
  if (!ok && t == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (t < 32) tmem_dealloc(tmem, 128);
}

// Sum the per-CTA gradients in CTA order and take one Adam step.
__global__ void mlp_adam_kernel(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                                const float* __restrict__ grad, int nblk, int step, float lr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  float g = 0.0f;
  for (int b = 0; b < nblk; ++b) g += grad[(long long)b * NPARAM + i];
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, (float)(step + 1)));
  const float vh = vi / (1.0f - powf(b2, (float)(step + 1)));
  P[i] -= lr * mh / (sqrtf(vh) + eps);
}

// Forward only, over given samples (the inference path without the cut construction): p, or with
// `correction` the correction s CORR (2p - 1) of the homogenized features.
__global__ void __launch_bounds__(TILE)
    mlp_predict_kernel(const float* __restrict__ P, const float* __restrict__ feats, long long n, int correction,
                       float* __restrict__ out, int* __restrict__ err, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem[];
  const MlpShared s = mlp_shared(smem, false, wait_limit);
  const int t = threadIdx.x;
  stage_weights(P, s, false);
  if (t == 0) mbar_init(s.mbar, 1);
  if (t < 32) { tmem_alloc(s.tmem, 64); tmem_relinquish(); }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem;
  uint32_t phase = 0;
  bool ok = true;
  for (long long base = (long long)blockIdx.x * TILE; base < n; base += (long long)gridDim.x * TILE) {
    const long long q = base + t;
    float xr[8], x[8], sc = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) xr[k] = q < n ? feats[q * 8 + k] : 0.0f;
    if (correction) homogenize(xr, x, sc);
    else {
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = xr[k];
    }
    float z;
    if (!mlp_forward(s, tmem, x, false, phase, z)) { ok = false; break; }
    if (q < n) {
      const float p = sigmoidf_(z);
      out[q] = correction ? sc * CORR * (2.0f * p - 1.0f) : p;
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok && t == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (t < 32) tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------------------------------------
// Fused cut-band kernel with the learned correction: each CTA takes tiles of 128 listed cut cells,
// one per thread, builds their plain moments (writing every field), then runs the network on the
// tile and replaces the volume fraction where the correction is accepted.
template <class T>
struct LearnedArgs {
  DevGrid<T> g;
  const T* phi;
  cci::Cols cols;
  DevTable tb;
  const unsigned* cut_list;
  const unsigned* cut_count;
  const float* P;
  float bound;
  unsigned long long* fallback;
  int* err;
  long long wait_limit;
};

// BUILD: the kernel builds each listed cell's plain moments itself; without it the plain cut-band
// kernel has already written them (mc_cut_kernel, the same construction at three times this
// kernel's occupancy) and this kernel only reads the plain fraction back and corrects it.
template <class T, bool BUILD>
__global__ void __launch_bounds__(TILE) mc_cut_learned_kernel(const LearnedArgs<T> A) {
  extern __shared__ __align__(128) unsigned char smem[];
  const MlpShared s = mlp_shared(smem, false, A.wait_limit);
  const int t = threadIdx.x;
  stage_weights(A.P, s, false);
  if (t == 0) mbar_init(s.mbar, 1);
  if (t < 32) { tmem_alloc(s.tmem, 64); tmem_relinquish(); }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem;
  uint32_t phase = 0;
  const long long n0 = A.g.n[0], n1 = A.g.n[1];
  const long long nx = n0 + 1, ny = n1 + 1;
  Stage<T> st;
  st.kind = A.cols.kind;
  st.amb = A.cols.amb;
  st.vf = static_cast<T*>(A.cols.vf);
  st.c = static_cast<T*>(A.cols.c);
  st.ff = static_cast<T*>(A.cols.ff);
  st.fcl = static_cast<T*>(A.cols.fcl);
  st.ic = static_cast<T*>(A.cols.ic);
  const T cs[3] = {A.g.d[0], A.g.d[1], A.g.d[2]};
  const float inv_h = 1.0f / float(A.g.d[0]);
  const long long total = *A.cut_count;
  unsigned long long fb = 0;
  bool ok = true;
  for (long long base = (long long)blockIdx.x * TILE; base < total; base += (long long)gridDim.x * TILE) {
    const long long q = base + t;
    float x[8] = {0, 0, 0, 0, 0, 0, 0, 0}, sc = 0.0f;
    long long ci = -1;
    T plain = T(0);
    if (q < total) {
      ci = A.cut_list[q];
      const long long i = ci % n0, j = (ci / n0) % n1, k = ci / (n0 * n1);
      const long long b0 = i + nx * (j + ny * k);
      const long long bz = nx * ny;
      const T ph[8] = {A.phi[b0], A.phi[b0 + 1], A.phi[b0 + nx + 1], A.phi[b0 + nx],
                       A.phi[b0 + bz], A.phi[b0 + bz + 1], A.phi[b0 + bz + nx + 1], A.phi[b0 + bz + nx]};
      if constexpr (BUILD) {
        const T org[3] = {node_coord(A.g.x0[0], A.g.d[0], i), node_coord(A.g.x0[1], A.g.d[1], j),
                          node_coord(A.g.x0[2], A.g.d[2], k)};
        const T l[3] = {node_coord(A.g.x0[0], A.g.d[0], i + 1) - org[0],
                        node_coord(A.g.x0[1], A.g.d[1], j + 1) - org[1],
                        node_coord(A.g.x0[2], A.g.d[2], k + 1) - org[2]};
        mc_cut_cell<T>(ph, l, org, cs, A.tb, st, ci);
      }
      plain = st.vf[ci];
      float xr[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) xr[c] = float(ph[c]) * inv_h;
      homogenize(xr, x, sc);
    }
    float z;
    if (!mlp_forward(s, tmem, x, false, phase, z)) { ok = false; break; }
    if (q < total) {
      const float p = sigmoidf_(z);
      const float corr = sc * CORR * (2.0f * p - 1.0f);
      const T v = plain + T(corr);
      const bool accept = isfinite(corr) && fabsf(corr) <= A.bound && v >= T(0) && v <= T(1);
      if (accept) st.vf[ci] = v;
      else ++fb;
    }
    tc_fence_before();
    __syncthreads();
  }
  if (fb) atomicAdd(A.fallback, fb);
  if (!ok && t == 0) atomicExch(A.err, 1);
  tc_fence_before();
  __syncthreads();
  if (t < 32) tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------------------------------------
// Training samples: for each listed cut cell, its features (8 corner phi / h), its plain volume
// fraction, its linear index and the label -- the fluid fraction marching cubes gives it at 8x
// sub-refinement: update_cache! on the one-cell grid CartesianGrid(get_node(g, cell), (8,8,8), d/8)
// (the idiom of test/test_mc_moments.jl:67-69,91-98), in Float64, its 512 fractions averaged. A
// sub-node is get_node of that grid, (x0 + T(i) d) + T(a) d/8. The sum runs in a fixed order:
// each thread's four sub-cells t, t+128, t+256, t+384, then a butterfly within each warp, then
// (w0 + w1) + (w2 + w3).
constexpr int LBL_NT = 128;
constexpr int LBL_SUB_BYTES = ((729 * 8 + 15) / 16) * 16;  // staged columns then start 16-byte aligned
__global__ void __launch_bounds__(LBL_NT) label_kernel(const DevGrid<double> g, const DevTape tape, const float* __restrict__ phi,
                                                      const float* __restrict__ vf, const DevTable tb,
                                                      const unsigned* __restrict__ list, long long n,
                                                      float* __restrict__ feats, float* __restrict__ labels,
                                                      float* __restrict__ plain, int64_t* __restrict__ index) {
  extern __shared__ __align__(128) unsigned char smem[];
  double* sub = reinterpret_cast<double*>(smem);                    // 729 sub-node values
  unsigned char* stg = smem + LBL_SUB_BYTES;                        // one cell slot per thread
  double* red = reinterpret_cast<double*>(stg + LBL_NT * 208);      // 4 partials
  unsigned char* tp = reinterpret_cast<unsigned char*>(red + 4);
  const STape<double> t = load_tape<double>(tape.bytes, tape.n_ops, tape.n_params, tp);
  __syncthreads();
  Stage<double> st;
  st.kind = reinterpret_cast<int8_t*>(stg);
  st.amb = stg + LBL_NT;
  st.vf = reinterpret_cast<double*>(stg + 2 * LBL_NT);
  st.c = st.vf + LBL_NT;
  st.ff = st.c + 3 * LBL_NT;
  st.fcl = st.ff + 6 * LBL_NT;
  st.ic = st.fcl + 12 * LBL_NT;
  const long long n0 = g.n[0], n1 = g.n[1];
  const long long nx = n0 + 1, ny = n1 + 1;
  const double sd[3] = {g.d[0] / 8.0, g.d[1] / 8.0, g.d[2] / 8.0};
  const float inv_hf = 1.0f / float(g.d[0]);
  for (long long q = blockIdx.x; q < n; q += gridDim.x) {
    const long long ci = list[q];
    const long long i = ci % n0, j = (ci / n0) % n1, k = ci / (n0 * n1);
    // the one-cell grid's origin: the cell's first node
    const double cx0[3] = {node_coord(g.x0[0], g.d[0], i), node_coord(g.x0[1], g.d[1], j),
                           node_coord(g.x0[2], g.d[2], k)};
    for (int v = threadIdx.x; v < 729; v += LBL_NT) {
      const int a = v % 9, b = (v / 9) % 9, c = v / 81;
      const double xyz[3] = {node_coord(cx0[0], sd[0], a), node_coord(cx0[1], sd[1], b),
                             node_coord(cx0[2], sd[2], c)};
      sub[v] = tape_eval<double, 3, double>(t, xyz);
    }
    __syncthreads();
    double acc = 0.0;
    for (int sc = threadIdx.x; sc < 512; sc += LBL_NT) {
      const int a = sc % 8, b = (sc / 8) % 8, c = sc / 64;
      const int s0 = a + 9 * (b + 9 * c);
      const double ph[8] = {sub[s0], sub[s0 + 1], sub[s0 + 10], sub[s0 + 9],
                            sub[s0 + 81], sub[s0 + 82], sub[s0 + 91], sub[s0 + 90]};
      int nout = 0;
#pragma unroll
      for (int e = 0; e < 8; ++e) nout += nudge(ph[e]) >= 0.0 ? 1 : 0;
      if (nout == 8) acc += 1.0;
      else if (nout > 0) {
        const double org[3] = {node_coord(cx0[0], sd[0], a), node_coord(cx0[1], sd[1], b),
                               node_coord(cx0[2], sd[2], c)};
        const double l[3] = {node_coord(cx0[0], sd[0], a + 1) - org[0], node_coord(cx0[1], sd[1], b + 1) - org[1],
                             node_coord(cx0[2], sd[2], c + 1) - org[2]};
        mc_cut_cell<double>(ph, l, org, sd, tb, st, threadIdx.x);
        acc += st.vf[threadIdx.x];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      labels[q] = float(((red[0] + red[1]) + (red[2] + red[3])) / 512.0);
      plain[q] = vf[ci];
      if (index) index[q] = ci;
    }
    if (threadIdx.x < 8) {
      const int e = threadIdx.x;
      const long long b0 = i + nx * (j + ny * k);
      const long long off[8] = {0, 1, nx + 1, nx, nx * ny, nx * ny + 1, nx * ny + nx + 1, nx * ny + nx};
      feats[q * 8 + e] = phi[b0 + off[e]] * inv_hf;  // as the learned update forms them
    }
    __syncthreads();
  }
}

}  // namespace

// =============================================================================================
namespace cci {

int mlp_nparam() { return NPARAM; }

template <class T>
cudaError_t launch_mc_cut_learned(const DevGrid<T>& g, const T* phi, const Cols& cols, const DevTable& tb,
                                  const unsigned* cut_list, const unsigned* cut_count, const float* P, float bound,
                                  unsigned long long* fallback, int* err, cudaStream_t s, bool build) {
  LearnedArgs<T> a{g, phi, cols, tb, cut_list, cut_count, P, bound, fallback, err, wait_limit()};
  const int sm = MlpLayout::INFER_SMEM;
  cudaError_t e;
  if (build) {
    e = cudaFuncSetAttribute(mc_cut_learned_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    mc_cut_learned_kernel<T, true><<<148 * 3, TILE, sm, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(mc_cut_learned_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    mc_cut_learned_kernel<T, false><<<148 * 3, TILE, sm, s>>>(a);
  }
  return cudaGetLastError();
}
template cudaError_t launch_mc_cut_learned<float>(const DevGrid<float>&, const float*, const Cols&, const DevTable&,
                                                  const unsigned*, const unsigned*, const float*, float,
                                                  unsigned long long*, int*, cudaStream_t, bool);
template cudaError_t launch_mc_cut_learned<double>(const DevGrid<double>&, const double*, const Cols&, const DevTable&,
                                                   const unsigned*, const unsigned*, const float*, float,
                                                   unsigned long long*, int*, cudaStream_t, bool);

// One training step's gradients: per-CTA partials in grad[tiles][NPARAM], per-CTA squared-error
// sums in loss[tiles].
cudaError_t launch_mlp_grads(const float* P, const float* feats, const float* labels, const float* plain,
                             const float* weights, long long n, unsigned long long seed, int step, int tiles,
                             bool augment, float* grad, float* loss, int* err, cudaStream_t s) {
  const int sm = MlpLayout::TRAIN_BYTES;
  cudaError_t e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  mlp_train_kernel<<<tiles, TILE, sm, s>>>(P, feats, labels, plain, weights, n, seed, step, augment ? 1 : 0,
                                           1.0f / float(tiles * TILE), grad, loss, err, wait_limit());
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* P, float* m, float* v, const float* grad, int tiles, int step, float lr,
                            cudaStream_t s) {
  mlp_adam_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(P, m, v, grad, tiles, step, lr);
  return cudaGetLastError();
}

cudaError_t launch_mlp_predict(const float* P, const float* feats, long long n, bool correction, float* out, int* err,
                               cudaStream_t s) {
  const int sm = MlpLayout::INFER_SMEM;
  cudaError_t e = cudaFuncSetAttribute(mlp_predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  long long tiles = (n + TILE - 1) / TILE;
  const int grid = (int)(tiles < 148 * 3 ? (tiles < 1 ? 1 : tiles) : 148 * 3);
  mlp_predict_kernel<<<grid, TILE, sm, s>>>(P, feats, n, correction ? 1 : 0, out, err, wait_limit());
  return cudaGetLastError();
}

cudaError_t launch_labels(const DevGrid<double>& g, const DevTape& tape, const float* phi, const float* vf,
                          const DevTable& tb, const unsigned* list, long long n, float* feats, float* labels,
                          float* plain, int64_t* index, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int sm = LBL_SUB_BYTES + LBL_NT * 208 + 4 * 8 + ((tape.bytes_len + 15) / 16) * 16;
  cudaError_t e = cudaFuncSetAttribute(label_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  const long long grid = n < 148 * 8 ? n : 148 * 8;
  label_kernel<<<(unsigned)grid, LBL_NT, sm, s>>>(g, tape, phi, vf, tb, list, n, feats, labels, plain, index);
  return cudaGetLastError();
}

}  // namespace cci
