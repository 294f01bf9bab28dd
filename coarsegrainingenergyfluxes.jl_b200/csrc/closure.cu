// Learned closure (no counterpart in the reference): a pointwise MLP 5 -> 64 -> 64 -> 64 -> 3
// with GELU, trained and evaluated on the 5th-generation tensor cores, and the judge that checks
// its flux against the exact path tile by tile.
//
// Tensor-core mapping.  One CTA of 128 threads owns a tile of 128 points: the points are the M = 128
// rows of every tcgen05.mma (cta_group::1, kind::f16, BF16 operands, FP32 accumulators in tensor
// memory), so thread t reads accumulator lane t back with tcgen05.ld.32x32b and finishes point t
// (bias, GELU, BF16 rounding) straight into the next layer's shared-memory operand.  Every operand is
// a K-major tile in the canonical no-swizzle layout (8 x 8 core matrices of 128 B; K-adjacent core
// matrices 128 B apart, row groups K/8 * 128 B apart).  One thread issues the MMAs of a step and
// commits them to an mbarrier that every thread waits on (bounded; a timeout sets an error flag).
// The weight gradients dW^T = H_prev^T dZ contract over the tile's points: their A operand is the
// transposed activation tile (input units as rows, the 128 points as K) and their FP32 accumulators
// stay in tensor memory across all tiles of the CTA; a row of ones under each transposed activation
// tile makes the same MMA produce the bias gradient.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "cgef_internal.h"

namespace cgef {
namespace {

constexpr int kNin = 5, kNh = 64, kNout = 3;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kNh * kNin, kOffW2 = kOffB1 + kNh, kOffB2 = kOffW2 + kNh * kNh,
              kOffW3 = kOffB2 + kNh, kOffB3 = kOffW3 + kNh * kNh, kOffW4 = kOffB3 + kNh,
              kOffB4 = kOffW4 + kNout * kNh, kNParam = kOffB4 + kNout;
static_assert(kNParam == CGEF_CLOSURE_NPARAM, "parameter layout");

// Packed operand image (bytes): BF16 K-major tiles exactly as the kernels hold them in shared
// memory, then the FP32 biases b1[64] b2[64] b3[64] b4[16].
constexpr int kImgW1 = 0;       // [64 x 16]  (inputs 5..15 zero)
constexpr int kImgW2 = 2048;    // [64 x 64]
constexpr int kImgW3 = 10240;   // [64 x 64]
constexpr int kImgW4 = 18432;   // [16 x 64]  (outputs 3..15 zero)
constexpr int kImgFwd = 20480;  // forward tiles end here
constexpr int kImgW2T = 20480;  // [64 x 64]  row = input unit, K = output unit
constexpr int kImgW3T = 28672;  // [64 x 64]
constexpr int kImgW4T = 36864;  // [64 x 16]
constexpr int kImgTiles = 38912;
constexpr int kBiasN = 208;
constexpr int kImgBytes = kImgTiles + kBiasN * 4;

constexpr int kTile = 128;
constexpr long long kWaitCycles = 4000000000LL;  // about 2 s at the B200's clocks

// Tensor-memory columns of the training kernel (512 allocated; one CTA per SM).
constexpr uint32_t kTZ1 = 0, kTZ2 = 64, kTZ3 = 128, kTDH = 192, kTDW1 = 256, kTDW2 = 320, kTDW3 = 384, kTY = 448,
                   kTDW4 = 464;
// Inference kernel: one reused 64-column pre-activation block and the outputs (128 allocated).
constexpr uint32_t kIZ = 0, kIY = 64;

// Byte offset of element (r, k) of a K-major tile with K columns (K a multiple of 8).
__host__ __device__ constexpr int kmaj(int r, int k, int K) {
  return (r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// ---- tcgen05 / mbarrier primitives ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, leading (K-direction) and stride (row-group) byte offsets,
// descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const long long start = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - start > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's accumulator lane; waits for the load.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// D (+)= A * B^T over `ksteps` K-slices of 16: A is M=128 rows (SBO a_sbo), B is N rows (SBO b_sbo),
// both K-major with 128 B between K-adjacent core matrices.
__device__ __forceinline__ void gemm(uint32_t tmem_d, uint32_t a, uint32_t a_sbo, uint32_t b, uint32_t b_sbo, int N,
                                     int ksteps, bool accumulate) {
  const uint32_t id = idesc_bf16(128, N);
  for (int s = 0; s < ksteps; ++s)
    mma_bf16(tmem_d, sdesc(a + 256u * s, 128u, a_sbo), sdesc(b + 256u * s, 128u, b_sbo), id,
             (accumulate || s > 0) ? 1u : 0u);
}

// One MMA step: publishes the threads' shared-memory writes to the tensor cores, lets thread 0
// issue, and waits (bounded) for completion.  Uniform result across the CTA.
template <class F>
__device__ __forceinline__ bool mma_step(uint32_t bar, uint32_t& phase, F issue) {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    issue();
    mma_commit(bar);
  }
  const bool mine = mbar_wait_bounded(bar, phase);
  phase ^= 1u;
  const bool ok = __syncthreads_and(mine ? 1 : 0) != 0;
  tc_fence_after();
  return ok;
}

// ---- numerics shared with the oracle (closure_oracle.c) ----
__device__ __forceinline__ float gelu(float a) { return 0.5f * a * (1.0f + erff(a * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float a) {
  return 0.5f * (1.0f + erff(a * 0.70710678118654752f)) + a * expf(-0.5f * a * a) * 0.39894228040143268f;
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Row r, columns c0..c0+15 of a K-major tile with K columns (BF16 rounding).
__device__ __forceinline__ void put_row16(uint8_t* buf, int K, int r, int c0, const float (&v)[16]) {
  uint4 q0 = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
  uint4 q1 = make_uint4(pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]), pack2(v[14], v[15]));
  *reinterpret_cast<uint4*>(buf + kmaj(r, c0, K)) = q0;
  *reinterpret_cast<uint4*>(buf + kmaj(r, c0 + 8, K)) = q1;
}

// Column r (a point), rows c0..c0+15 (units) of a transposed tile with the 128 points as K.
__device__ __forceinline__ void put_col16(uint8_t* buf, int r, int c0, const float (&v)[16]) {
#pragma unroll
  for (int i = 0; i < 16; ++i)
    *reinterpret_cast<__nv_bfloat16*>(buf + kmaj(c0 + i, r, kTile)) = __float2bfloat16_rn(v[i]);
}

__device__ __forceinline__ void put_bf16(uint8_t* buf, int off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(buf + off) = __float2bfloat16_rn(v);
}

// Forward epilogue: h = GELU(z + b) for the 64 units of this thread's point.
__device__ __forceinline__ void epi_forward(uint32_t tz, const float* bias, uint8_t* sH, uint8_t* sHT) {
  const int p = threadIdx.x;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    float v[16];
    tmem_load16(tz + 16 * c, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + bias[16 * c + i]);
    put_row16(sH, kNh, p, 16 * c, v);
    if (sHT) put_col16(sHT, p, 16 * c, v);
  }
}

// Backward epilogue: dz = dh * GELU'(z + b).
__device__ __forceinline__ void epi_backward(uint32_t tdh, uint32_t tz, const float* bias, uint8_t* sDZ,
                                             uint8_t* sDZT) {
  const int p = threadIdx.x;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    float dh[16], z[16];
    tmem_load16(tdh + 16 * c, dh);
    tmem_load16(tz + 16 * c, z);
#pragma unroll
    for (int i = 0; i < 16; ++i) dh[i] = dh[i] * gelu_grad(z[i] + bias[16 * c + i]);
    if (sDZ) put_row16(sDZ, kNh, p, 16 * c, dh);
    put_col16(sDZT, p, 16 * c, dh);
  }
}

// ---- training: forward + backward over a batch, per-CTA gradient partials ----
struct TrainK {
  const uint8_t* image;  // kImgBytes
  const float* x;        // [count][5]
  const float* t;        // [count][3]
  int64_t count;
  float inv_count;
  float* gpart;  // [gridDim.x][kNParam]
  float* lpart;  // [gridDim.x]
  int* err;
};

// Shared-memory map of the training kernel (bytes).  The transposed activation tiles XT, H1T, H2T,
// H3T lie back to back and are followed by DZ, so an M = 128 MMA reading any of them stays inside
// the allocation (the rows past a tile's own are read and their accumulator lanes ignored).
constexpr int kSXT = 0, kSH1T = 4096, kSH2T = 22528, kSH3T = 40960, kSDZ = 59392, kSDZT = 75776, kSW = 92160,
              kSX = 131072, kSH = 135168, kSDY = 151552, kSDYT = 155648, kSBias = 159744, kSRed = 160576,
              kSBar = 160640, kSTmem = 160648, kTrainSmem = 160768;
static_assert(kSW + kImgTiles == kSX, "training smem map");
static_assert(kSH3T + 128 * 256 <= kSDZT, "M = 128 reads of H3T stay in DZ");

__global__ void __launch_bounds__(128, 1) closure_train_kernel(TrainK a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sXT = sm + kSXT;
  uint8_t* sH1T = sm + kSH1T;
  uint8_t* sH2T = sm + kSH2T;
  uint8_t* sH3T = sm + kSH3T;
  uint8_t* sDZ = sm + kSDZ;
  uint8_t* sDZT = sm + kSDZT;
  uint8_t* sW = sm + kSW;
  uint8_t* sX = sm + kSX;
  uint8_t* sH = sm + kSH;
  uint8_t* sDY = sm + kSDY;
  uint8_t* sDYT = sm + kSDYT;
  float* sB = reinterpret_cast<float*>(sm + kSBias);
  float* sRed = reinterpret_cast<float*>(sm + kSRed);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < kImgTiles / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(sW)[i] = reinterpret_cast<const uint4*>(a.image)[i];
  for (int i = tid; i < kBiasN; i += blockDim.x) sB[i] = reinterpret_cast<const float*>(a.image + kImgTiles)[i];
  {
    // constant rows: XT row 5 and the H_lT row 64 are ones (bias gradients), the rest of their
    // row groups and DYT rows 3..15 are zero
    const int p = tid;
    for (int r = kNin; r < 16; ++r) put_bf16(sXT, kmaj(r, p, kTile), r == kNin ? 1.0f : 0.0f);
    for (int r = kNh; r < kNh + 8; ++r) {
      const float v = r == kNh ? 1.0f : 0.0f;
      put_bf16(sH1T, kmaj(r, p, kTile), v);
      put_bf16(sH2T, kmaj(r, p, kTile), v);
      put_bf16(sH3T, kmaj(r, p, kTile), v);
    }
    for (int r = kNout; r < 16; ++r) put_bf16(sDYT, kmaj(r, p, kTile), 0.0f);
  }
  const uint32_t bar = smem_u32(sm + kSBar);
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(smem_u32(sm + kSTmem), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tb = *reinterpret_cast<volatile uint32_t*>(sm + kSTmem);
  const uint32_t trow = tb + (static_cast<uint32_t>(warp * 32) << 16);

  const uint32_t uXT = smem_u32(sXT), uH1T = smem_u32(sH1T), uH2T = smem_u32(sH2T), uH3T = smem_u32(sH3T);
  const uint32_t uDZ = smem_u32(sDZ), uDZT = smem_u32(sDZT), uX = smem_u32(sX), uH = smem_u32(sH);
  const uint32_t uDY = smem_u32(sDY), uDYT = smem_u32(sDYT);
  const uint32_t uW1 = smem_u32(sW + kImgW1), uW2 = smem_u32(sW + kImgW2), uW3 = smem_u32(sW + kImgW3),
                 uW4 = smem_u32(sW + kImgW4), uW2T = smem_u32(sW + kImgW2T), uW3T = smem_u32(sW + kImgW3T),
                 uW4T = smem_u32(sW + kImgW4T);

  uint32_t phase = 0;
  bool ok = true;
  int done = 0;
  float lsum = 0.0f;
  const int64_t ntiles = (a.count + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t q = tile * kTile + tid;
    const bool valid = q < a.count;
    float xf[16], tg[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 16; ++k) xf[k] = 0.0f;
    if (valid) {
#pragma unroll
      for (int k = 0; k < kNin; ++k) xf[k] = a.x[q * kNin + k];
#pragma unroll
      for (int o = 0; o < kNout; ++o) tg[o] = a.t[q * kNout + o];
    }
    put_row16(sX, 16, tid, 0, xf);
#pragma unroll
    for (int k = 0; k < kNin; ++k) put_bf16(sXT, kmaj(k, tid, kTile), xf[k]);

    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kTZ1, uX, 256, uW1, 256, 64, 1, false); }))) break;
    epi_forward(trow + kTZ1, sB, sH, sH1T);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kTZ2, uH, 1024, uW2, 1024, 64, 4, false); }))) break;
    epi_forward(trow + kTZ2, sB + 64, sH, sH2T);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kTZ3, uH, 1024, uW3, 1024, 64, 4, false); }))) break;
    epi_forward(trow + kTZ3, sB + 128, sH, sH3T);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kTY, uH, 1024, uW4, 1024, 16, 4, false); }))) break;
    {
      float y[16], dy[16];
      tmem_load16(trow + kTY, y);
#pragma unroll
      for (int o = 0; o < 16; ++o) dy[o] = 0.0f;
      if (valid) {
#pragma unroll
        for (int o = 0; o < kNout; ++o) {
          const float e = (y[o] + sB[192 + o]) - tg[o];
          lsum += e * e;
          dy[o] = 2.0f * e * a.inv_count;
        }
      }
      put_row16(sDY, 16, tid, 0, dy);
#pragma unroll
      for (int o = 0; o < kNout; ++o) put_bf16(sDYT, kmaj(o, tid, kTile), dy[o]);
    }
    const bool acc = done > 0;
    if (!(ok = mma_step(bar, phase, [&] {
          gemm(tb + kTDW4, uH3T, 2048, uDYT, 2048, 16, 8, acc);
          gemm(tb + kTDH, uDY, 256, uW4T, 256, 64, 1, false);
        })))
      break;
    epi_backward(trow + kTDH, trow + kTZ3, sB + 128, sDZ, sDZT);
    if (!(ok = mma_step(bar, phase, [&] {
          gemm(tb + kTDW3, uH2T, 2048, uDZT, 2048, 64, 8, acc);
          gemm(tb + kTDH, uDZ, 1024, uW3T, 1024, 64, 4, false);
        })))
      break;
    epi_backward(trow + kTDH, trow + kTZ2, sB + 64, sDZ, sDZT);
    if (!(ok = mma_step(bar, phase, [&] {
          gemm(tb + kTDW2, uH1T, 2048, uDZT, 2048, 64, 8, acc);
          gemm(tb + kTDH, uDZ, 1024, uW2T, 1024, 64, 4, false);
        })))
      break;
    epi_backward(trow + kTDH, trow + kTZ1, sB, nullptr, sDZT);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kTDW1, uXT, 2048, uDZT, 2048, 64, 8, acc); }))) break;
    ++done;
  }

  if (ok) {
    // accumulator lane r = input index r of the layer (r == fan_in: the bias), column = output unit
    float* gp = a.gpart + static_cast<int64_t>(blockIdx.x) * kNParam;
    const int r = tid;
    const float keep = done > 0 ? 1.0f : 0.0f;
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_load16(trow + kTDW1 + 16 * c, v);
      for (int i = 0; i < 16; ++i) {
        const int o = 16 * c + i;
        if (r < kNin) gp[kOffW1 + o * kNin + r] = keep * v[i];
        else if (r == kNin) gp[kOffB1 + o] = keep * v[i];
      }
    }
    const uint32_t cols[2] = {kTDW2, kTDW3};
    const int offw[2] = {kOffW2, kOffW3}, offb[2] = {kOffB2, kOffB3};
    for (int l = 0; l < 2; ++l)
      for (int c = 0; c < 4; ++c) {
        float v[16];
        tmem_load16(trow + cols[l] + 16 * c, v);
        for (int i = 0; i < 16; ++i) {
          const int o = 16 * c + i;
          if (r < kNh) gp[offw[l] + o * kNh + r] = keep * v[i];
          else if (r == kNh) gp[offb[l] + o] = keep * v[i];
        }
      }
    {
      float v[16];
      tmem_load16(trow + kTDW4, v);
      for (int o = 0; o < kNout; ++o) {
        if (r < kNh) gp[kOffW4 + o * kNh + r] = keep * v[o];
        else if (r == kNh) gp[kOffB4 + o] = keep * v[o];
      }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if (lane == 0) sRed[warp] = lsum;
    __syncthreads();
    if (tid == 0) a.lpart[blockIdx.x] = sRed[0] + sRed[1] + sRed[2] + sRed[3];
  } else {
    // an MMA step did not complete in time: flag it, give the outstanding step one more bounded
    // wait, and release tensor memory
    if (tid == 0) atomicExch(a.err, 1);
    mbar_wait_bounded(bar, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tb, 512);
}

// ---- inference: features -> MLP -> tau -> Pi, persistent over tiles ----
struct InferK {
  const uint8_t* image;
  const float* x_in;     // raw features [N][5] (forward mode) or nullptr
  float* y_out;          // raw outputs [N][3] (forward mode) or nullptr
  const float* grad;     // [nb][4][N] ell^2-scaled gradient components
  const double* gmean;   // [nb] mean |grad|^2 over active points
  const uint8_t* mask;
  int64_t mask_stride;
  int64_t N;
  int64_t tiles_per_slice;
  int64_t ntiles;
  float logfeat;
  double inv_l2;  // 1 / ell^2
  void* pi;
  int dtype;
  int* err;
};

constexpr int kIW = 0, kIX = 20480, kIH = 24576, kIBias = 40960, kIBar = 41792, kITmem = 41800;
// requested dynamic shared memory: at most four CTAs per SM, so four 128-column tensor-memory
// allocations never exceed the SM's 512 columns
constexpr int kInferSmem = 55296;

__global__ void __launch_bounds__(128) closure_infer_kernel(InferK a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sW = sm + kIW;
  uint8_t* sX = sm + kIX;
  uint8_t* sH = sm + kIH;
  float* sB = reinterpret_cast<float*>(sm + kIBias);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < kImgFwd / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(sW)[i] = reinterpret_cast<const uint4*>(a.image)[i];
  for (int i = tid; i < kBiasN; i += blockDim.x) sB[i] = reinterpret_cast<const float*>(a.image + kImgTiles)[i];
  const uint32_t bar = smem_u32(sm + kIBar);
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(smem_u32(sm + kITmem), 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tb = *reinterpret_cast<volatile uint32_t*>(sm + kITmem);
  const uint32_t trow = tb + (static_cast<uint32_t>(warp * 32) << 16);
  const uint32_t uX = smem_u32(sX), uH = smem_u32(sH);
  const uint32_t uW1 = smem_u32(sW + kImgW1), uW2 = smem_u32(sW + kImgW2), uW3 = smem_u32(sW + kImgW3),
                 uW4 = smem_u32(sW + kImgW4);
  uint32_t phase = 0;
  bool ok = true;
  for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int64_t s = tile / a.tiles_per_slice;
    const int64_t q = (tile - s * a.tiles_per_slice) * kTile + tid;
    const bool valid = q < a.N;
    float f[16], g[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.0f;
    bool act = false;
    double gm = 0.0;
    if (valid) {
      if (a.x_in) {
        act = true;
#pragma unroll
        for (int k = 0; k < kNin; ++k) f[k] = a.x_in[q * kNin + k];
      } else {
        act = a.mask == nullptr || a.mask[s * a.mask_stride + q] != 0;
        gm = a.gmean[s];
        const float inv = gm > 0.0 ? static_cast<float>(1.0 / sqrt(gm)) : 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) g[k] = a.grad[(s * 4 + k) * a.N + q];
        if (act) {
#pragma unroll
          for (int k = 0; k < 4; ++k) f[k] = g[k] * inv;
          f[4] = a.logfeat;
        }
      }
    }
    put_row16(sX, 16, tid, 0, f);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kIZ, uX, 256, uW1, 256, 64, 1, false); }))) break;
    epi_forward(trow + kIZ, sB, sH, nullptr);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kIZ, uH, 1024, uW2, 1024, 64, 4, false); }))) break;
    epi_forward(trow + kIZ, sB + 64, sH, nullptr);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kIZ, uH, 1024, uW3, 1024, 64, 4, false); }))) break;
    epi_forward(trow + kIZ, sB + 128, sH, nullptr);
    if (!(ok = mma_step(bar, phase, [&] { gemm(tb + kIY, uH, 1024, uW4, 1024, 16, 4, false); }))) break;
    float yv[16];
    tmem_load16(trow + kIY, yv);
    float y[3];
#pragma unroll
    for (int o = 0; o < kNout; ++o) y[o] = yv[o] + sB[192 + o];
    if (valid && a.y_out) {
#pragma unroll
      for (int o = 0; o < kNout; ++o) a.y_out[q * kNout + o] = y[o];
    }
    if (valid && a.pi) {
      double pi = 0.0;
      if (act) {
        const double sc = gm * a.inv_l2;  // n^2 / ell^2
        const double tee = y[0] * sc, ten = y[1] * sc, tnn = y[2] * sc;
        const double see = g[0] * a.inv_l2, sen = 0.5 * (static_cast<double>(g[1]) + g[2]) * a.inv_l2,
                     snn = g[3] * a.inv_l2;
        pi = -(see * tee + 2.0 * sen * ten + snn * tnn);
      }
      if (a.dtype == CGEF_F32)
        static_cast<float*>(a.pi)[s * a.N + q] = static_cast<float>(pi);
      else
        static_cast<double*>(a.pi)[s * a.N + q] = pi;
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(a.err, 1);
    mbar_wait_bounded(bar, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tb, 128);
}

// ---- optimiser and operand packing ----
__device__ void pack_param(uint8_t* img, int i, float p) {
  float* bias = reinterpret_cast<float*>(img + kImgTiles);
  if (i < kOffB1) {
    const int o = i / kNin, k = i % kNin;
    put_bf16(img, kImgW1 + kmaj(o, k, 16), p);
  } else if (i < kOffW2) {
    bias[i - kOffB1] = p;
  } else if (i < kOffB2) {
    const int o = (i - kOffW2) / kNh, k = (i - kOffW2) % kNh;
    put_bf16(img, kImgW2 + kmaj(o, k, kNh), p);
    put_bf16(img, kImgW2T + kmaj(k, o, kNh), p);
  } else if (i < kOffW3) {
    bias[64 + i - kOffB2] = p;
  } else if (i < kOffB3) {
    const int o = (i - kOffW3) / kNh, k = (i - kOffW3) % kNh;
    put_bf16(img, kImgW3 + kmaj(o, k, kNh), p);
    put_bf16(img, kImgW3T + kmaj(k, o, kNh), p);
  } else if (i < kOffW4) {
    bias[128 + i - kOffB3] = p;
  } else if (i < kOffB4) {
    const int o = (i - kOffW4) / kNh, k = (i - kOffW4) % kNh;
    put_bf16(img, kImgW4 + kmaj(o, k, kNh), p);
    put_bf16(img, kImgW4T + kmaj(k, o, 16), p);
  } else {
    bias[192 + i - kOffB4] = p;
  }
}

__device__ __forceinline__ bool is_bias(int i) {
  return (i >= kOffB1 && i < kOffW2) || (i >= kOffB2 && i < kOffW3) || (i >= kOffB3 && i < kOffW4) || i >= kOffB4;
}

struct AdamK {
  float* params;
  float* m;
  float* v;
  const float* gpart;
  const float* lpart;
  int nparts;
  int step;
  float lr, b1, b2, eps, wd;
  uint8_t* image;
  float* loss_out;  // may be null
  float loss_scale;  // 1 / batch points
  float* grad_out;  // gradient mode: write the summed gradient, no update
};

__global__ void closure_adamw_kernel(AdamK a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && a.loss_out) {
    float l = 0.0f;
    for (int c = 0; c < a.nparts; ++c) l += a.lpart[c];
    *a.loss_out = l * a.loss_scale;
  }
  if (i >= kNParam) return;
  float g = 0.0f;
  for (int c = 0; c < a.nparts; ++c) g += a.gpart[static_cast<int64_t>(c) * kNParam + i];
  if (a.grad_out) {
    a.grad_out[i] = g;
    return;
  }
  const float c1 = 1.0f - powf(a.b1, static_cast<float>(a.step)), c2 = 1.0f - powf(a.b2, static_cast<float>(a.step));
  const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
  const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
  a.m[i] = m;
  a.v[i] = v;
  float p = a.params[i];
  if (!is_bias(i)) p -= a.lr * a.wd * p;
  p = p - a.lr * (m / c1) / (sqrtf(v / c2) + a.eps);
  a.params[i] = p;
  pack_param(a.image, i, p);
}

__global__ void closure_pack_kernel(const float* params, uint8_t* image) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kNParam) pack_param(image, i, params[i]);
}

// ---- closure support kernels ----
// Planetary (X, Y, Z) filtered velocity -> local east/north components.
__global__ void rotate_local_kernel(const double* V, int64_t vstride, double* ub, int64_t ustride, const double* sinlam,
                                    const double* coslam, const double* sinphi, const double* cosphi, int nx, int ny) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int s = blockIdx.z;
  if (i >= nx) return;
  const int64_t N = static_cast<int64_t>(nx) * ny, pix = static_cast<int64_t>(j) * nx + i;
  const double* v = V + s * vstride + pix;
  const double X = v[0], Y = v[N], Z = v[2 * N];
  const double sl = sinlam[i], cl = coslam[i], sp = sinphi[j], cp = cosphi[j];
  ub[s * ustride + pix] = -sl * X + cl * Y;
  ub[s * ustride + N + pix] = -sp * cl * X - sp * sl * Y + cp * Z;
}

// Training pairs from the ell^2-scaled gradients and the exact local tau.
__global__ void pairs_kernel(const float* grad, const double* gmean, const double* gather, int64_t gstride,
                             const uint8_t* mask, int64_t mstride, int64_t N, float logfeat, double l2, float* feat,
                             float* targ) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (q >= N) return;
  const bool act = mask == nullptr || mask[s * mstride + q] != 0;
  const double gm = gmean[s];
  const double inv = gm > 0.0 ? 1.0 / sqrt(gm) : 0.0;
  const double tsc = gm > 0.0 ? l2 / gm : 0.0;
  float* fo = feat + static_cast<int64_t>(s) * 5 * N + q;
  float* to = targ + static_cast<int64_t>(s) * 3 * N + q;
  for (int k = 0; k < 4; ++k) fo[k * N] = act ? static_cast<float>(grad[(static_cast<int64_t>(s) * 4 + k) * N + q] * inv) : 0.0f;
  fo[4 * N] = act ? logfeat : 0.0f;
  const double* g = gather + s * gstride + q;
  for (int o = 0; o < 3; ++o) to[o * N] = act ? static_cast<float>(g[(2 + o) * N] * tsc) : 0.0f;
}

// One block per (judged tile, slice): exact Pi from the exact tau and the closure's gradients;
// accumulates the closure's squared error and the exact squared flux, then writes the exact value.
__global__ void judge_kernel(const int32_t* tiles, int ntiles, const double* gather, int64_t gstride, const float* grad,
                             const uint8_t* mask, int64_t mstride, int nx, int ny, double inv_l2, void* pi, int dtype,
                             double* sums) {
  __shared__ double sd[256], se[256];
  const int t = blockIdx.x, s = blockIdx.y;
  const int tx = tiles[2 * t], ty = tiles[2 * t + 1];
  const int64_t N = static_cast<int64_t>(nx) * ny;
  double d2 = 0.0, e2 = 0.0;
  for (int k = threadIdx.x; k < 32 * 32; k += blockDim.x) {
    const int i = tx * 32 + (k & 31), j = ty * 32 + (k >> 5);
    if (i >= nx || j >= ny) continue;
    const int64_t q = static_cast<int64_t>(j) * nx + i;
    if (!(mask == nullptr || mask[s * mstride + q] != 0)) continue;
    const float* g = grad + static_cast<int64_t>(s) * 4 * N + q;
    const double* G = gather + s * gstride + q;
    const double see = g[0] * inv_l2, sen = 0.5 * (static_cast<double>(g[N]) + g[2 * N]) * inv_l2, snn = g[3 * N] * inv_l2;
    const double pe = -(see * G[2 * N] + 2.0 * sen * G[3 * N] + snn * G[4 * N]);
    const int64_t o = static_cast<int64_t>(s) * N + q;
    double pm;
    if (dtype == CGEF_F32) {
      pm = static_cast<float*>(pi)[o];
      static_cast<float*>(pi)[o] = static_cast<float>(pe);
    } else {
      pm = static_cast<double*>(pi)[o];
      static_cast<double*>(pi)[o] = pe;
    }
    d2 += (pm - pe) * (pm - pe);
    e2 += pe * pe;
  }
  sd[threadIdx.x] = d2;
  se[threadIdx.x] = e2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) {
      sd[threadIdx.x] += sd[threadIdx.x + w];
      se[threadIdx.x] += se[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[(static_cast<int64_t>(s) * ntiles + t) * 2] = sd[0];
    sums[(static_cast<int64_t>(s) * ntiles + t) * 2 + 1] = se[0];
  }
}

int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

constexpr double kLogEllC = 12.317637;  // ln(223607 m): geometric centre of 50..1000 km
constexpr double kLogEllH = 1.4978661;  // ln(20) / 2

float log_feature(double ell) { return static_cast<float>((std::log(ell) - kLogEllC) / kLogEllH); }

}  // namespace
}  // namespace cgef

using namespace cgef;

struct cgef_closure {
  int device = -1;
  int sms = 148;
  float* d_params = nullptr;
  float* d_m = nullptr;
  float* d_v = nullptr;
  uint8_t* d_image = nullptr;
  float* d_gpart = nullptr;
  float* d_lpart = nullptr;
  int* d_err = nullptr;
  int64_t step = 0;
  DeviceBuffer ws[6];  // 0 ub/vb, 1 grad planes, 2 gmean + partials, 3 judge tiles + sums, 4 exact pi scratch
};

namespace {

int cl_ws(cgef_closure* c, int slot, size_t bytes, void** out) {
  DeviceBuffer& b = c->ws[slot];
  if (b.bytes < bytes) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CGEF_ENOMEM, "closure workspace allocation failed");
    }
    b.bytes = bytes;
  }
  *out = b.ptr;
  return CGEF_OK;
}

int check_closure(const cgef_closure* c) {
  if (!c) return fail(CGEF_EINVAL, "closure is NULL");
  return CGEF_OK;
}

// The error word a kernel sets when a bounded wait runs out: reported as CGEF_ETIMEOUT, then cleared
// so that the closure's next call starts clean (the wait's kernel released its tensor memory and
// returned; the context stays usable).
int read_err(cgef_closure* c, cudaStream_t st) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "closure error flag");
  if (h) {
    e = cudaMemsetAsync(c->d_err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "closure error flag reset");
    return fail(CGEF_ETIMEOUT, "a closure tensor-core step did not complete within its wait limit");
  }
  return CGEF_OK;
}

// Runs the training kernel over `count` points; the AdamW kernel then either updates (grad_out
// null) or writes the summed gradient.
int train_pass(cgef_closure* c, const float* x, const float* t, int64_t count, const cgef_adamw* opt, float* loss,
               float* grad_out, cudaStream_t st) {
  const int64_t ntiles = (count + kTile - 1) / kTile;
  const int grid = static_cast<int>(std::min<int64_t>(ntiles, c->sms));
  TrainK k{c->d_image, x, t, count, 1.0f / static_cast<float>(count), c->d_gpart, c->d_lpart, c->d_err};
  prof_begin(CGEF_KERNEL_CLOSURE, st);
  closure_train_kernel<<<grid, 128, kTrainSmem, st>>>(k);
  prof_end(CGEF_KERNEL_CLOSURE, st);
  int rc = launch_check("closure_train_kernel");
  if (rc) return rc;
  AdamK a{};
  a.params = c->d_params;
  a.m = c->d_m;
  a.v = c->d_v;
  a.gpart = c->d_gpart;
  a.lpart = c->d_lpart;
  a.nparts = grid;
  a.image = c->d_image;
  a.loss_out = loss;
  a.loss_scale = 1.0f / static_cast<float>(count);
  a.grad_out = grad_out;
  if (!grad_out) {
    a.step = static_cast<int>(++c->step);
    a.lr = static_cast<float>(opt->lr);
    a.b1 = static_cast<float>(opt->beta1);
    a.b2 = static_cast<float>(opt->beta2);
    a.eps = static_cast<float>(opt->eps);
    a.wd = static_cast<float>(opt->weight_decay);
  }
  closure_adamw_kernel<<<(kNParam + 255) / 256, 256, 0, st>>>(a);
  return launch_check("closure_adamw_kernel");
}

// Filtered local velocity (ubar, vbar planes, FP64) of nbatch slices through the plan's engine;
// also leaves the staged input planes in the plan's slot for a later exact pass.
int filtered_velocity(cgef_plan* p, cgef_closure* c, int dtype, const void* u, const void* v, int nbatch,
                      const uint8_t* mask, int64_t mstride, double** ubvb, double** planes_out, int* pitch_out,
                      int* np_out, cudaStream_t st) {
  int rc;
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = stage_pi(p, dtype, u, v, nbatch, mask, mstride, p->H, &planes, &pitch, &np, st))) return rc;
  void* uv = nullptr;
  if ((rc = cl_ws(c, 0, sizeof(double) * 2 * N * nbatch, &uv))) return rc;
  double* UV = static_cast<double*>(uv);
  const bool sph = p->geometry == CGEF_SPHERICAL;
  const int nf = sph ? 3 : 2;
  double* out = UV;
  if (sph) {
    void* vp = nullptr;
    if ((rc = ensure_ws(p, kSlotVel, sizeof(double) * 3 * N * nbatch, &vp))) return rc;
    out = static_cast<double*>(vp);
  }
  GatherOut go{};
  for (int m = 0; m < nf; ++m) go.o[m] = out + m * N;
  go.slice_stride = nf * N;
  const bool def = p->strategy == CGEF_DEFORMABLE;
  if (p->engine == CGEF_ENGINE_BANDED) {
    void* part = nullptr;
    const size_t pb = banded_scratch_bytes(p, nf + (def ? 1 : 0), nbatch, kModeFields);
    if (pb > 0 && (rc = ensure_ws(p, kSlotSplit, pb, &part))) return rc;
    rc = launch_banded(p, kModeFields, nf, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(part), go, st);
  } else if (p->engine == CGEF_ENGINE_SEPARABLE) {
    void* rb = nullptr;
    if ((rc = ensure_ws(p, kSlotAux, sizeof(double) * (nf + 1) * N * nbatch, &rb))) return rc;
    rc = launch_separable(p, kModeFields, nf, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(rb), go, st);
  } else {
    void* pre = nullptr;
    if ((rc = ensure_ws(p, kSlotAux, sizeof(double) * (nf + 1) * static_cast<int64_t>(p->ny) * (p->pre_ne + 1) * nbatch,
                        &pre)))
      return rc;
    rc = launch_prefix(p, kModeFields, nf, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(pre), go, st);
  }
  if (rc) return rc;
  if (sph) {
    dim3 grid((p->nx + 127) / 128, p->ny, nbatch);
    rotate_local_kernel<<<grid, 128, 0, st>>>(out, 3 * N, UV, 2 * N, p->d_sinlam, p->d_coslam, p->d_sinphi,
                                              p->d_cosphi, p->nx, p->ny);
    if ((rc = launch_check("rotate_local_kernel"))) return rc;
  }
  *ubvb = UV;
  *planes_out = planes;
  *pitch_out = pitch;
  *np_out = np;
  return CGEF_OK;
}

// ell^2-scaled gradient planes and their per-slice mean square from ubar/vbar planes (stride 2N or
// the 5-plane gather stride), optionally passing tau through.
int gradients(cgef_plan* p, cgef_closure* c, const double* ub, const double* vb, int64_t in_stride, int nbatch,
              const uint8_t* mask, int64_t mstride, float** grad, double** gmean, cudaStream_t st) {
  int rc;
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  void* gp = nullptr;
  if ((rc = cl_ws(c, 1, sizeof(float) * 4 * N * nbatch, &gp))) return rc;
  const int64_t nblk = strain_tiles(p);
  void* gm = nullptr;
  if ((rc = cl_ws(c, 2, sizeof(double) * (nbatch + 2 * nblk * nbatch), &gm))) return rc;
  StrainArgs sa{};
  sa.ubar = ub;
  sa.vbar = vb;
  sa.in_slice_stride = in_stride;
  sa.mask = mask;
  sa.mask_slice_stride = mstride;
  sa.nbatch = nbatch;
  sa.dtype = CGEF_F64;
  sa.out_slice_stride = N;
  sa.grad = static_cast<float*>(gp);
  sa.grad_slice_stride = 4 * N;
  sa.grad_scale = p->scale * p->scale;
  sa.grad_mean = static_cast<double*>(gm);
  sa.grad_partials = static_cast<double*>(gm) + nbatch;
  if ((rc = launch_strain(p, sa, st))) return rc;
  *grad = static_cast<float*>(gp);
  *gmean = static_cast<double*>(gm);
  return CGEF_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

int cgef::closure_inject_timeout(cgef_closure* c) {
  if (!c) return fail(CGEF_EINVAL, "closure is NULL");
  const int one = 1;
  cudaError_t e = cudaMemcpy(c->d_err, &one, sizeof(int), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "closure error word");
}

extern "C" {

int32_t cgef_closure_create(cgef_closure** out, uint64_t seed) {
  if (!out) return fail(CGEF_EINVAL, "out is NULL");
  *out = nullptr;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(CGEF_ENODEVICE, "no CUDA device");
  }
  cgef_closure* c = new (std::nothrow) cgef_closure();
  if (!c) return fail(CGEF_ENOMEM, "closure allocation failed");
  c->device = dev;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return fail(CGEF_ENODEVICE, "cannot query the CUDA device");
  }
  c->sms = prop.multiProcessorCount;
  if (prop.major < 10) {
    delete c;
    return fail(CGEF_EUNSUPPORTED, "the closure's tensor-core kernels need an sm_100 device");
  }
  const int maxparts = c->sms;
  cudaError_t e = cudaMalloc(&c->d_params, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_m, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_v, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_image, kImgBytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_gpart, sizeof(float) * kNParam * maxparts);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_lpart, sizeof(float) * maxparts);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_m, 0, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMemset(c->d_v, 0, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMemset(c->d_image, 0, kImgBytes);
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(closure_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 kTrainSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(closure_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 kInferSmem);
  if (e != cudaSuccess) {
    cgef_closure_destroy(c);
    return cuda_fail(e, "closure setup");
  }
  // PyTorch-style uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) initialisation from the seed
  std::vector<float> P(kNParam);
  uint64_t s = seed;
  auto uni = [&](double bound) { return static_cast<float>(((splitmix(s) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * bound); };
  const double b1 = 1.0 / std::sqrt(double(kNin)), bh = 1.0 / std::sqrt(double(kNh));
  for (int i = 0; i < kNParam; ++i) P[i] = uni(i < kOffW2 ? b1 : bh);
  int rc = cgef_closure_set_params(c, P.data());
  if (rc) {
    cgef_closure_destroy(c);
    return rc;
  }
  *out = c;
  return CGEF_OK;
}

int32_t cgef_closure_destroy(cgef_closure* c) {
  if (!c) return CGEF_OK;
  DeviceGuard dg(c->device);
  cudaFree(c->d_params);
  cudaFree(c->d_m);
  cudaFree(c->d_v);
  cudaFree(c->d_image);
  cudaFree(c->d_gpart);
  cudaFree(c->d_lpart);
  cudaFree(c->d_err);
  for (auto& b : c->ws)
    if (b.ptr) cudaFree(b.ptr);
  delete c;
  return CGEF_OK;
}

int32_t cgef_closure_get_params(const cgef_closure* c, float* params) {
  int rc = check_closure(c);
  if (rc) return rc;
  if (!params) return fail(CGEF_EINVAL, "params is NULL");
  DeviceGuard dg(c->device);
  cudaError_t e = cudaMemcpy(params, c->d_params, sizeof(float) * kNParam, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "closure params D2H");
}

int32_t cgef_closure_set_params(cgef_closure* c, const float* params) {
  int rc = check_closure(c);
  if (rc) return rc;
  if (!params) return fail(CGEF_EINVAL, "params is NULL");
  DeviceGuard dg(c->device);
  cudaError_t e = cudaMemcpy(c->d_params, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->d_m, 0, sizeof(float) * kNParam);
  if (e == cudaSuccess) e = cudaMemset(c->d_v, 0, sizeof(float) * kNParam);
  if (e != cudaSuccess) return cuda_fail(e, "closure params H2D");
  c->step = 0;
  closure_pack_kernel<<<(kNParam + 255) / 256, 256>>>(c->d_params, c->d_image);
  if ((rc = launch_check("closure_pack_kernel"))) return rc;
  e = cudaDeviceSynchronize();
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "closure pack");
}

int32_t cgef_closure_train_device(cgef_closure* c, const float* x, const float* t, int64_t npoints, int64_t batch,
                                  int32_t nsteps, const cgef_adamw* opt, float* losses, void* stream) {
  int rc = check_closure(c);
  if (rc) return rc;
  if (!x || !t || !opt) return fail(CGEF_EINVAL, "x, t and opt must be non-NULL");
  if (npoints < 1 || batch < 1 || nsteps < 0) return fail(CGEF_EINVAL, "npoints, batch >= 1 and nsteps >= 0");
  DeviceGuard dg(c->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int k = 0; k < nsteps; ++k) {
    const int64_t start = (static_cast<int64_t>(k) * batch) % npoints;
    const int64_t count = std::min(batch, npoints - start);
    if ((rc = train_pass(c, x + start * kNin, t + start * kNout, count, opt, losses ? losses + k : nullptr, nullptr,
                         st)))
      return rc;
  }
  return read_err(c, st);
}

int32_t cgef_closure_grad_device(cgef_closure* c, const float* x, const float* t, int64_t npoints, float* grads,
                                 float* loss, void* stream) {
  int rc = check_closure(c);
  if (rc) return rc;
  if (!x || !t || !grads || !loss) return fail(CGEF_EINVAL, "x, t, grads and loss must be non-NULL");
  if (npoints < 1) return fail(CGEF_EINVAL, "npoints must be >= 1");
  DeviceGuard dg(c->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((rc = train_pass(c, x, t, npoints, nullptr, loss, grads, st))) return rc;
  return read_err(c, st);
}

int32_t cgef_closure_forward_device(cgef_closure* c, const float* x, int64_t npoints, float* y, void* stream) {
  int rc = check_closure(c);
  if (rc) return rc;
  if (!x || !y || npoints < 1) return fail(CGEF_EINVAL, "x, y must be non-NULL and npoints >= 1");
  DeviceGuard dg(c->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  InferK k{};
  k.image = c->d_image;
  k.x_in = x;
  k.y_out = y;
  k.N = npoints;
  k.tiles_per_slice = (npoints + kTile - 1) / kTile;
  k.ntiles = k.tiles_per_slice;
  k.err = c->d_err;
  const int grid = static_cast<int>(std::min<int64_t>(k.ntiles, static_cast<int64_t>(c->sms) * 4));
  prof_begin(CGEF_KERNEL_CLOSURE, st);
  closure_infer_kernel<<<grid, 128, kInferSmem, st>>>(k);
  prof_end(CGEF_KERNEL_CLOSURE, st);
  if ((rc = launch_check("closure_infer_kernel"))) return rc;
  return read_err(c, st);
}

int32_t cgef_closure_pairs_device(cgef_plan* p, int32_t dtype, const void* u, const void* v, int64_t nbatch64,
                                  const uint8_t* slice_masks, float* features, float* targets, void* stream) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (p->engine == CGEF_ENGINE_SPECTRAL) return fail(CGEF_EUNSUPPORTED, "the learned closure runs on real-space plans");
  if (!u || !v || !features || !targets) return fail(CGEF_EINVAL, "u, v, features and targets must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p->d_mask;
  const int64_t mstride = slice_masks ? N : 0;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = stage_pi(p, dtype, u, v, nbatch, mask, mstride, p->H, &planes, &pitch, &np, st))) return rc;
  void* gather = nullptr;
  if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
  double* G = static_cast<double*>(gather);
  if ((rc = pi_gather(p, planes, pitch, p->H, np, nbatch, mask, mstride, G, st))) return rc;
  // a throwaway closure workspace: the features need only the plan
  cgef_closure tmp;
  tmp.device = p->device;
  float* grad = nullptr;
  double* gmean = nullptr;
  rc = gradients(p, &tmp, G, G + N, 5 * N, nbatch, mask, mstride, &grad, &gmean, st);
  if (rc == CGEF_OK) {
    dim3 grid(static_cast<unsigned>((N + 255) / 256), nbatch);
    pairs_kernel<<<grid, 256, 0, st>>>(grad, gmean, G, 5 * N, mask, mstride, N, log_feature(p->scale),
                                       p->scale * p->scale, features, targets);
    rc = launch_check("pairs_kernel");
    if (rc == CGEF_OK) {
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) rc = cuda_fail(e, "closure pairs");
    }
  }
  for (auto& b : tmp.ws)
    if (b.ptr) cudaFree(b.ptr);
  for (auto& b : tmp.ws) b.ptr = nullptr;
  return rc;
}

int32_t cgef_closure_pi_device(cgef_closure* c, cgef_plan* p, int32_t dtype, const void* u, const void* v,
                               int64_t nbatch64, const uint8_t* slice_masks, double judge_fraction, uint64_t judge_seed,
                               double tol, void* pi, cgef_closure_report* report, void* stream) {
  int rc;
  if ((rc = check_closure(c)) || (rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (p->engine == CGEF_ENGINE_SPECTRAL) return fail(CGEF_EUNSUPPORTED, "the learned closure runs on real-space plans");
  if (!u || !v || !pi) return fail(CGEF_EINVAL, "u, v and pi must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  if (!(judge_fraction >= 0.0 && judge_fraction <= 1.0)) return fail(CGEF_EINVAL, "judge_fraction must be in [0, 1]");
  if (c->device != p->device) return fail(CGEF_EINVAL, "closure and plan live on different devices");
  DeviceGuard dg(p->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p->d_mask;
  const int64_t mstride = slice_masks ? N : 0;

  // 1. filtered velocity, gradients, closure flux
  double* UV = nullptr;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = filtered_velocity(p, c, dtype, u, v, nbatch, mask, mstride, &UV, &planes, &pitch, &np, st))) return rc;
  float* grad = nullptr;
  double* gmean = nullptr;
  if ((rc = gradients(p, c, UV, UV + N, 2 * N, nbatch, mask, mstride, &grad, &gmean, st))) return rc;
  InferK k{};
  k.image = c->d_image;
  k.grad = grad;
  k.gmean = gmean;
  k.mask = mask;
  k.mask_stride = mstride;
  k.N = N;
  k.tiles_per_slice = (N + kTile - 1) / kTile;
  k.ntiles = k.tiles_per_slice * nbatch;
  k.logfeat = log_feature(p->scale);
  k.inv_l2 = 1.0 / (p->scale * p->scale);
  k.pi = pi;
  k.dtype = dtype;
  k.err = c->d_err;
  const int grid = static_cast<int>(std::min<int64_t>(k.ntiles, static_cast<int64_t>(c->sms) * 4));
  prof_begin(CGEF_KERNEL_CLOSURE, st);
  closure_infer_kernel<<<grid, 128, kInferSmem, st>>>(k);
  prof_end(CGEF_KERNEL_CLOSURE, st);
  if ((rc = launch_check("closure_infer_kernel"))) return rc;

  // 2. judge: seeded tiles recomputed by the exact path
  const int ntx = (p->nx + 31) / 32, nty = (p->ny + 31) / 32, nt = ntx * nty;
  int nj = judge_fraction > 0.0 ? std::max(1, static_cast<int>(std::lround(judge_fraction * nt))) : 0;
  nj = std::min(nj, nt);
  cgef_closure_report rep{};
  if (nj > 0) {
    std::vector<int32_t> order(nt);
    for (int i = 0; i < nt; ++i) order[i] = i;
    uint64_t sd = judge_seed;
    for (int i = 0; i < nj; ++i) {
      const int r = i + static_cast<int>(splitmix(sd) % static_cast<uint64_t>(nt - i));
      std::swap(order[i], order[r]);
    }
    std::sort(order.begin(), order.begin() + nj);
    std::vector<int32_t> tiles(2 * nj);
    for (int i = 0; i < nj; ++i) {
      tiles[2 * i] = order[i] % ntx;
      tiles[2 * i + 1] = order[i] / ntx;
    }
    // exact tau at the judged tiles (banded: only their work items; other engines: everywhere)
    void* gather = nullptr;
    if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
    double* G = static_cast<double*>(gather);
    const int mode = mode_for(p);
    // a schedule of the judged tiles' work items alone, split finely enough to fill the GPU in
    // one wave (a few tiles cut at the whole grid's granularity would leave most SMs idle)
    std::vector<WorkItem> items;
    std::vector<SplitGroup> groups;
    int jslots = 0;
    const bool banded = p->engine == CGEF_ENGINE_BANDED;
    if (banded) {
      std::vector<std::pair<int, int>> tl(nj);
      for (int i = 0; i < nj; ++i) tl[i] = {tiles[2 * i], tiles[2 * i + 1]};
      subset_schedule(p, tl, c->sms, items, groups, jslots);
    }
    const size_t tiles_b = sizeof(int32_t) * 2 * nj, items_b = sizeof(WorkItem) * items.size();
    const size_t groups_b = sizeof(SplitGroup) * groups.size();
    const size_t sums_b = sizeof(double) * 2 * static_cast<size_t>(nj) * nbatch;
    auto al = [](size_t b) { return (b + 15) / 16 * 16; };
    void* jw = nullptr;
    if ((rc = cl_ws(c, 3, al(sums_b) + al(tiles_b) + al(items_b) + al(groups_b) + 16, &jw))) return rc;
    char* jb = static_cast<char*>(jw);
    double* d_sums = reinterpret_cast<double*>(jb);
    int32_t* d_tiles = reinterpret_cast<int32_t*>(jb + al(sums_b));
    WorkItem* d_items = reinterpret_cast<WorkItem*>(jb + al(sums_b) + al(tiles_b));
    SplitGroup* d_groups = reinterpret_cast<SplitGroup*>(jb + al(sums_b) + al(tiles_b) + al(items_b));
    cudaError_t e = cudaMemcpyAsync(d_tiles, tiles.data(), tiles_b, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !items.empty())
      e = cudaMemcpyAsync(d_items, items.data(), items_b, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !groups.empty())
      e = cudaMemcpyAsync(d_groups, groups.data(), groups_b, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "judge tiles H2D");
    GatherOut go{};
    for (int m = 0; m < 5; ++m) go.o[m] = G + m * N;
    go.slice_stride = 5 * N;
    if (banded) {
      const int na = (mode == kModePiSphere ? 9 : 5) + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
      void* part = nullptr;
      const size_t pb = sizeof(double) * static_cast<size_t>(jslots) * nbatch * kRows * na * 32;
      if (pb > 0 && (rc = ensure_ws(p, kSlotSplit, pb, &part))) return rc;
      rc = launch_banded_items(p, mode, 0, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(part),
                               d_items, static_cast<int>(items.size()), d_groups, static_cast<int>(groups.size()), go,
                               st);
    } else
      rc = pi_gather(p, planes, pitch, p->H, np, nbatch, mask, mstride, G, st);
    if (rc) return rc;
    judge_kernel<<<dim3(nj, nbatch), 256, 0, st>>>(d_tiles, nj, G, 5 * N, grad, mask, mstride, p->nx, p->ny,
                                                   1.0 / (p->scale * p->scale), pi, dtype, d_sums);
    if ((rc = launch_check("judge_kernel"))) return rc;
    std::vector<double> sums(2 * static_cast<size_t>(nj) * nbatch);
    e = cudaMemcpyAsync(sums.data(), d_sums, sums_b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "judge sums");
    if ((rc = read_err(c, st))) return rc;
    for (int s = 0; s < nbatch; ++s) {
      double d2 = 0.0, e2 = 0.0;
      for (int i = 0; i < nj; ++i) {
        const double td = sums[(static_cast<size_t>(s) * nj + i) * 2], te = sums[(static_cast<size_t>(s) * nj + i) * 2 + 1];
        d2 += td;
        e2 += te;
        if (te > 0.0 ? std::sqrt(td / te) > tol : td > 0.0) ++rep.failed_tiles;
      }
      rep.judged_tiles += nj;
      const double est = e2 > 0.0 ? std::sqrt(d2 / e2) : (d2 > 0.0 ? INFINITY : 0.0);
      rep.est_rel_l2 = std::max(rep.est_rel_l2, est);
      if (est > tol) {
        // the judged error is above the tolerance: this slice takes the exact path
        const size_t fb = dsize(dtype) * static_cast<size_t>(N);
        cgef_pi_outputs o{};
        o.pi = static_cast<char*>(pi) + fb * s;
        const uint8_t* ms = slice_masks ? slice_masks + N * s : nullptr;
        if ((rc = compute_pi_device(p, dtype, static_cast<const char*>(u) + fb * s,
                                    static_cast<const char*>(v) + fb * s, 1, ms, &o, st)))
          return rc;
        ++rep.fallbacks;
      }
    }
  } else if ((rc = read_err(c, st))) {
    return rc;
  }
  if (report) *report = rep;
  return CGEF_OK;
}

}  // extern "C"
