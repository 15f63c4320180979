// Training of the soft-shadow denoiser on the library's own kernels.
//
// One step is: the forward pass (the inference kernels of denoise.cu on the
// float32 master weights rounded to FP16), the loss and its gradient at the
// sigmoid outputs, the backward pass, and an Adam update of the masters.
// Backward, per op in reverse order (G[b]: gradient of buffer b, FP16 NHWC,
// scaled by kLossScale):
//   convolution: dZ = G[out] * (out > 0) (or the loss gradient for the last
//     op); weight gradient dW = sum over pixels of dZ (x) the shifted input
//     (k_wgrad_tc, tcgen05); G[in] += conv(dZ, flipped transposed weights)
//     (the forward kernel, epilogue mode 3);
//   pooling: G[in] += G[out] spread over each 2x2 block / its pixel count;
//   upsample-add: G[skip] += G[out]; G[coarse] += G[out] summed per block.
// This is an extension with no counterpart in the reference.

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rtrace_gpu.h"
#include "denoise.hpp"

namespace rtb {
namespace {

constexpr float kLossScale = 256.0f;  // FP16 gradients: scaled sums, divided out in the Adam step
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle (the layout of
// denoise.cu's operands): start, leading byte offset between the two
// 8-element K halves of one MMA, stride byte offset between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16, FP32 accumulate, FP16 A and B, both K-major
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// 8 pixels x 8 channels (v[i]: the channels of pixel i) -> 8 channels x 8
// pixels (o[e]: channel e of pixels 0..7), FP16.
__device__ __forceinline__ void transpose8x8(const uint4 (&v)[8], uint4 (&o)[8]) {
#pragma unroll
  for (int e = 0; e < 8; e++) {
    const uint32_t sel = (e & 1) ? 0x7632u : 0x5410u;
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t a = (&v[2 * k].x)[e >> 1], b = (&v[2 * k + 1].x)[e >> 1];
      w[k] = __byte_perm(a, b, sel);
    }
    o[e] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

constexpr int WG_THREADS = 128;
constexpr int WG_TILE = 128;  // pixels of one row per step (the GEMM's K per step)

// Weight gradient of a 3x3 convolution with dilation `dil`:
//   dW[co][tap][ci] += sum over pixels q of dZ[q][co] * X[q + offset(tap)][ci]
// (zero outside the image), and the bias gradient db[co] += sum dZ[q][co].
// As GEMMs on the tensor cores: D[(tap, ci)][co] = A B with
//   A = the shifted inputs, M = 9 * CIN rows (tap, ci) in blocks of 128,
//       K = the 128 pixels of one step, and
//   B = dZ, N = COUT, the same K;
// one FP32 accumulator of COUT columns per M block stays in tensor memory
// for all the steps a CTA takes (steps: one 128-pixel run of one row).  The
// 128 threads stage operands in the K-major core-matrix layout (8 pixels x 8
// channels per thread, transposed in registers); thread 0 issues the MMAs
// and commits them to an mbarrier, which the stagers wait on before they
// overwrite the operands.  The epilogue adds the accumulators into dW with
// FP32 atomics.  Waits are bounded; one that runs out sets err and the CTA
// stops issuing.
template <int CIN, int COUT>
__global__ void __launch_bounds__(WG_THREADS) k_wgrad_tc(const __half* __restrict__ X, const __half* __restrict__ dZ,
                                                         int planes, int H, int W, int dil, float* __restrict__ dW,
                                                         float* __restrict__ db, int* err) {
  constexpr int MROWS = 9 * CIN;
  constexpr int NB = (MROWS + 127) / 128;  // M blocks
  constexpr int COLS = NB * COUT;
  constexpr int TMEM_ALLOC = COLS <= 32 ? 32 : COLS <= 64 ? 64 : COLS <= 128 ? 128 : COLS <= 256 ? 256 : 512;
  constexpr int A_BYTES = 16 * 2048;       // 128 rows x 128 pixels
  constexpr int B_BYTES = 16 * COUT * 16;  // COUT rows x 128 pixels
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* base = smem_raw + pad;
  unsigned char* sA = base;
  unsigned char* sB = base + A_BYTES;
  unsigned char* tail = sB + B_BYTES;
  const uint32_t bar = smem_u32(tail);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tail + 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tail + 12);
  float* s_db = reinterpret_cast<float*>(tail + 16);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < COUT; i += WG_THREADS) s_db[i] = 0.f;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_ALLOC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t IDESC = umma_idesc(128, COUT);
  const int tiles_x = (W + WG_TILE - 1) / WG_TILE;
  const long long nsteps = (long long)planes * H * tiles_x;
  uint32_t phase = 0;
  long long issued = 0;  // MMA groups committed (each followed by one wait)
  bool first = true;     // the accumulators still hold garbage
  const uint4 zero = make_uint4(0, 0, 0, 0);
  for (long long st = blockIdx.x; st < nsteps && !*abort_flag; st += gridDim.x) {
    const int tx = (int)(st % tiles_x);
    long long q = st / tiles_x;
    const int y = (int)(q % H);
    const long long p = q / H;
    const int x0 = tx * WG_TILE;
    for (int m = 0; m < NB; m++) {
      // the MMAs of the previous group have read the operands
      if (issued > 0) {
        if (!mbar_wait(bar, phase)) {
          if (tid == 0) atomicOr(err, DN_ERR_WAIT);
          *abort_flag = 1;
        }
        phase ^= 1u;
        issued = 0;
      }
      __syncthreads();
      if (*abort_flag) break;
      if (m == 0) {
        // B: dZ of this run, rows co, K = pixels; units (8 channels, 8 pixels)
        for (int u = tid; u < (COUT / 8) * 16; u += WG_THREADS) {
          const int c8 = u % (COUT / 8), g = u / (COUT / 8);
          uint4 v[8], o[8];
          float sum[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int x = x0 + 8 * g + i;
            v[i] = x < W ? reinterpret_cast<const uint4*>(dZ + ((p * H + y) * (long long)W + x) * COUT)[c8] : zero;
            const __half2* h = reinterpret_cast<const __half2*>(&v[i]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float2 f = __half22float2(h[k]);
              sum[2 * k] += f.x;
              sum[2 * k + 1] += f.y;
            }
          }
          transpose8x8(v, o);
          uint4* dst = reinterpret_cast<uint4*>(sB + g * (COUT * 16) + c8 * 128);
#pragma unroll
          for (int e = 0; e < 8; e++) dst[e] = o[e];
#pragma unroll
          for (int e = 0; e < 8; e++) atomicAdd(&s_db[8 * c8 + e], sum[e]);
        }
      }
      // A block m: rows r = m * 128 + j, (tap, ci) = (r / CIN, r % CIN)
      for (int u = tid; u < 16 * 16; u += WG_THREADS) {
        const int a8 = u % 16, g = u / 16;  // row group (8 rows), pixel group
        const int r0 = m * 128 + 8 * a8;
        uint4 v[8], o[8];
        if (r0 < MROWS) {
          const int tap = r0 / CIN, c8 = (r0 % CIN) / 8;
          const int yy = y + (tap / 3 - 1) * dil;
          const int xs = x0 + 8 * g + (tap % 3 - 1) * dil;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int x = xs + i;
            const bool in = yy >= 0 && yy < H && x >= 0 && x < W && x0 + 8 * g + i < W;
            v[i] = in ? reinterpret_cast<const uint4*>(X + ((p * H + yy) * (long long)W + x) * CIN)[c8] : zero;
          }
          transpose8x8(v, o);
        } else {
#pragma unroll
          for (int e = 0; e < 8; e++) o[e] = zero;
        }
        uint4* dst = reinterpret_cast<uint4*>(sA + g * 2048 + a8 * 128);
#pragma unroll
        for (int e = 0; e < 8; e++) dst[e] = o[e];
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(m * COUT);
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
        for (int s2 = 0; s2 < WG_TILE / 16; s2++) {
          const uint64_t da = umma_desc(a0 + (uint32_t)(2 * s2 * 2048), 2048, 128);
          const uint64_t dbd = umma_desc(b0 + (uint32_t)(2 * s2 * COUT * 16), COUT * 16, 128);
          const uint32_t accum = (first && s2 == 0) ? 0u : 1u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
              "}\n" ::"r"(acc),
              "l"(da), "l"(dbd), "r"(IDESC), "r"(accum)
              : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                     : "memory");
      }
      issued = 1;
    }
    first = false;
  }
  // drain the last group
  if (issued > 0 && !*abort_flag) {
    if (!mbar_wait(bar, phase)) {
      if (tid == 0) atomicOr(err, DN_ERR_WAIT);
      *abort_flag = 1;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!first && !*abort_flag) {
    // thread tid <-> accumulator row (lane) tid of each block
    for (int m = 0; m < NB; m++) {
      const int r = m * 128 + tid;
#pragma unroll
      for (int c0 = 0; c0 < COUT; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + (uint32_t)(m * COUT + c0) + ((uint32_t)(warp * 32) << 16), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (r < MROWS) {
          const int tap = r / CIN, ci = r % CIN;
#pragma unroll
          for (int k = 0; k < 16; k++) atomicAdd(&dW[((size_t)(c0 + k) * 9 + tap) * CIN + ci], __uint_as_float(v[k]));
        }
      }
    }
    for (int i = tid; i < COUT; i += WG_THREADS) atomicAdd(&db[i], s_db[i]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_ALLOC) : "memory");
  }
}

template <int CIN, int COUT>
cudaError_t launch_wgrad(const __half* X, const __half* dZ, int planes, int H, int W, int dil, float* dW, float* db,
                         int* err, cudaStream_t s, int num_sms) {
  const int smem = 1024 + 16 * 2048 + 16 * COUT * 16 + 16 + 4 * 64;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 64 || !attr_set[dev]) {
    e = cudaFuncSetAttribute(k_wgrad_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set[dev] = true;
  }
  const long long nsteps = (long long)planes * H * ((W + WG_TILE - 1) / WG_TILE);
  const int grid = (int)std::max<long long>(1, std::min<long long>(nsteps, num_sms));
  k_wgrad_tc<CIN, COUT><<<grid, WG_THREADS, smem, s>>>(X, dZ, planes, H, W, dil, dW, db, err);
  return cudaGetLastError();
}

// ---- elementwise kernels of the backward pass (8 FP16 channels a thread)
__device__ __forceinline__ void h8_to_f(const uint4& v, float (&f)[8]) {
  const __half2* h = reinterpret_cast<const __half2*>(&v);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float2 t = __half22float2(h[k]);
    f[2 * k] = t.x;
    f[2 * k + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 f_to_h8(const float (&f)[8]) {
  uint4 v;
  __half2* h = reinterpret_cast<__half2*>(&v);
#pragma unroll
  for (int k = 0; k < 4; k++) h[k] = __floats2half2_rn(f[2 * k], f[2 * k + 1]);
  return v;
}

#define RTB_GRID_STRIDE(t, n) \
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (n); t += (long long)gridDim.x * blockDim.x)

// dst = (first ? 0 : dst) + src
__global__ void k_acc(__half* dst, const __half* src, long long n8, int first) {
  RTB_GRID_STRIDE(t, n8) {
    float a[8], b[8];
    h8_to_f(reinterpret_cast<const uint4*>(src)[t], b);
    if (!first) {
      h8_to_f(reinterpret_cast<const uint4*>(dst)[t], a);
#pragma unroll
      for (int k = 0; k < 8; k++) b[k] += a[k];
    }
    reinterpret_cast<uint4*>(dst)[t] = f_to_h8(b);
  }
}

// out = g * (y > 0)
__global__ void k_relu_mask(const __half* g, const __half* y, __half* out, long long n8) {
  RTB_GRID_STRIDE(t, n8) {
    float a[8], b[8];
    h8_to_f(reinterpret_cast<const uint4*>(g)[t], a);
    h8_to_f(reinterpret_cast<const uint4*>(y)[t], b);
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = b[k] > 0.f ? a[k] : 0.f;
    reinterpret_cast<uint4*>(out)[t] = f_to_h8(a);
  }
}

// Adjoint of 2x2 average pooling: gin(y, x) (+)= gout(y/2, x/2) / count of
// the block's pixels inside the image.  gin [P][H][W][C], gout at half size.
__global__ void k_pool_adj(const __half* gout, __half* gin, int P, int H, int W, int C, int first) {
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2, CC = C / 8;
  const long long n = (long long)P * H * W * CC;
  RTB_GRID_STRIDE(t, n) {
    const int cc = (int)(t % CC);
    long long q = t / CC;
    const int x = (int)(q % W);
    q /= W;
    const int y = (int)(q % H);
    const long long p = q / H;
    const int by = y / 2, bx = x / 2;
    const int cnt = (min(2 * by + 2, H) - 2 * by) * (min(2 * bx + 2, W) - 2 * bx);
    float g[8], a[8];
    h8_to_f(reinterpret_cast<const uint4*>(gout + ((p * Ho + by) * (long long)Wo + bx) * C)[cc], g);
    const float inv = 1.f / (float)cnt;
    if (!first) h8_to_f(reinterpret_cast<const uint4*>(gin)[t], a);
#pragma unroll
    for (int k = 0; k < 8; k++) g[k] = g[k] * inv + (first ? 0.f : a[k]);
    reinterpret_cast<uint4*>(gin)[t] = f_to_h8(g);
  }
}

// Adjoint of nearest 2x upsampling: glow(y, x) (+)= sum of gout over the
// 2x2 block (pixels inside the image).  gout [P][H][W][C], glow half size.
__global__ void k_downsum(const __half* gout, __half* glow, int P, int H, int W, int C, int first) {
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2, CC = C / 8;
  const long long n = (long long)P * Ho * Wo * CC;
  RTB_GRID_STRIDE(t, n) {
    const int cc = (int)(t % CC);
    long long q = t / CC;
    const int x = (int)(q % Wo);
    q /= Wo;
    const int y = (int)(q % Ho);
    const long long p = q / Ho;
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, g[8];
    for (int dy = 0; dy < 2; dy++)
      for (int dx = 0; dx < 2; dx++) {
        const int yy = 2 * y + dy, xx = 2 * x + dx;
        if (yy >= H || xx >= W) continue;
        h8_to_f(reinterpret_cast<const uint4*>(gout + ((p * H + yy) * (long long)W + xx) * C)[cc], g);
#pragma unroll
        for (int k = 0; k < 8; k++) s[k] += g[k];
      }
    if (!first) {
      h8_to_f(reinterpret_cast<const uint4*>(glow)[t], g);
#pragma unroll
      for (int k = 0; k < 8; k++) s[k] += g[k];
    }
    reinterpret_cast<uint4*>(glow)[t] = f_to_h8(s);
  }
}

// Loss at the sigmoid outputs over the masked samples (the primary sample
// hit and the slot's light exists): sum of (v - t)^2 + (c - |v - t|)^2, the
// second term not differentiated through v.  Writes the scaled gradient
// with respect to the last convolution's pre-activation outputs (16 FP16
// channels; 0-1 visibility, 2-3 error estimate, the rest zero), and adds
// the masked count and the two loss sums to acc[0..2].
__global__ void k_loss(const float* vis, const float* conf, const __half* target, const __half* feat, __half* dz,
                       int P, int H, int W, float* acc) {
  const long long n = (long long)P * H * W;
  const long long plane = (long long)H * W;
  float cnt = 0.f, lv = 0.f, lc = 0.f;
  RTB_GRID_STRIDE(t, n) {
    const long long p = t / plane, pix = t % plane;
    const __half* f = feat + t * FEAT_CHANNELS;
    const bool valid = __half2float(f[FEAT_VALID]) > 0.f;
    float g[16];
#pragma unroll
    for (int k = 0; k < 16; k++) g[k] = 0.f;
    for (int j = 0; j < DN_MAX_SLOTS; j++) {
      const bool present = __half2float(f[FEAT_SLOT0 + FEAT_SLOT_STRIDE * j + 3]) > 0.f;
      if (!valid || !present) continue;
      const long long o = (p * DN_MAX_SLOTS + j) * plane + pix;
      const float v = vis[o], c = conf[o], tg = __half2float(target[o]);
      const float e = v - tg, ae = fabsf(e);
      cnt += 1.f;
      lv += e * e;
      lc += (c - ae) * (c - ae);
      g[j] = kLossScale * 2.f * e * v * (1.f - v);
      g[DN_MAX_SLOTS + j] = kLossScale * 2.f * (c - ae) * c * (1.f - c);
    }
    uint4* d = reinterpret_cast<uint4*>(dz + t * 16);
    float a[8], b[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      a[k] = g[k];
      b[k] = g[8 + k];
    }
    d[0] = f_to_h8(a);
    d[1] = f_to_h8(b);
  }
  for (int off = 16; off > 0; off >>= 1) {
    cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    lv += __shfl_down_sync(0xffffffffu, lv, off);
    lc += __shfl_down_sync(0xffffffffu, lc, off);
  }
  if ((threadIdx.x & 31) == 0 && cnt > 0.f) {
    atomicAdd(&acc[0], cnt);
    atomicAdd(&acc[1], lv);
    atomicAdd(&acc[2], lc);
  }
}

// Non-finite gradient entries (an FP16 activation gradient that overflowed
// the loss scale) into acc[3].
__global__ void k_grad_check(const float* grad, long long n, float* acc) {
  float bad = 0.f;
  RTB_GRID_STRIDE(i, n) bad += isfinite(grad[i]) ? 0.f : 1.f;
  for (int off = 16; off > 0; off >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, off);
  if ((threadIdx.x & 31) == 0 && bad > 0.f) atomicAdd(&acc[3], bad);
}

// Adam on the FP32 masters (weights [cout][3][3][cin] then bias, per
// convolution, concatenated): g = grad / (loss scale * masked count).  A
// step whose gradient has a non-finite entry (acc[3] > 0) is skipped.
__global__ void k_adam(float* w, float* m, float* v, const float* grad, long long n, const float* acc, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  if (acc[3] > 0.f) return;
  const float denom = kLossScale * fmaxf(acc[0], 1.f);
  RTB_GRID_STRIDE(i, n) {
    const float g = grad[i] / denom;
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// FP32 master weights [cout][3][3][cin] -> the FP16 operand layouts of the
// forward convolution (rows co, K = (tap, ci)) and of its backward data
// pass (rows ci, K = (tap, co) with the taps mirrored: the transposed
// convolution), element (n, k) at (k / 8) * (N * 8) + n * 8 + k % 8.
__global__ void k_pack_weights(const float* w, int cin, int cout, __half* fwd, __half* bwd) {
  const long long n = (long long)cout * 9 * cin;
  RTB_GRID_STRIDE(t, n) {
    const int ci = (int)(t % cin);
    const int tap = (int)((t / cin) % 9);
    const int co = (int)(t / (9 * cin));
    const __half h = __float2half_rn(w[t]);
    const int kf = tap * cin + ci;
    fwd[(size_t)(kf / 8) * (cout * 8) + co * 8 + kf % 8] = h;
    const int kb = (8 - tap) * cout + co;
    bwd[(size_t)(kb / 8) * (cin * 8) + ci * 8 + kb % 8] = h;
  }
}

int grid_for(long long n, int num_sms) {
  return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)num_sms * 16));
}
int level_dim(int n, int level) { return (n + (1 << level) - 1) >> level; }

}  // namespace

cudaError_t wgrad_launch(int cin, int cout, const __half* X, const __half* dZ, int planes, int H, int W, int dil,
                         float* dW, float* db, int* err, cudaStream_t s, int num_sms) {
#define RTB_WG(CI, CO) \
  if (cin == CI && cout == CO) return launch_wgrad<CI, CO>(X, dZ, planes, H, W, dil, dW, db, err, s, num_sms);
  RTB_WG(16, 16)
  RTB_WG(16, 32)
  RTB_WG(32, 16)
  RTB_WG(32, 32)
  RTB_WG(32, 64)
  RTB_WG(64, 32)
  RTB_WG(64, 64)
#undef RTB_WG
  return cudaErrorInvalidValue;
}

}  // namespace rtb

using namespace rtb;

// The trainer: master weights and Adam moments, the per-op FP16 weight
// layouts, activations and gradients for a fixed batch shape.
struct rt_dn_trainer {
  rt_ctx* ctx = nullptr;
  DenoiseNet net;  // forward weights point into fwd
  int planes = 0, H = 0, W = 0;
  std::vector<int> conv_of_op;       // op -> index among convolutions, -1 otherwise
  std::vector<size_t> woff;          // per convolution: offset of its weights in the flat master array
  std::vector<__half*> wbwd;         // per convolution: backward-data operand layout
  std::vector<void*> allocs;
  float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *acc = nullptr, *zeros = nullptr;
  long long n_params = 0;
  __half *arena = nullptr, *gbuf = nullptr, *dz = nullptr, *tmp = nullptr;
  std::vector<size_t> act_off, g_off;  // per buffer (1..n): offsets in arena / gbuf (halves)
  float *vis = nullptr, *conf = nullptr;
  int* err = nullptr;
  long long steps = 0;
  std::vector<unsigned char> blob_head;  // the loaded blob's ops, for export
};

namespace rtb {
// Host side of the C ABI (render.cu holds the context internals).
cudaStream_t ctx_stream(rt_ctx* ctx);
int ctx_device(rt_ctx* ctx);
int ctx_num_sms(rt_ctx* ctx);
rt_status ctx_fail(rt_ctx* ctx, rt_status st, const std::string& msg);
}  // namespace rtb

namespace {
template <class T>
cudaError_t talloc(rt_dn_trainer* t, T** p, size_t n) {
  *p = nullptr;
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) t->allocs.push_back(*p);
  return e;
}

void trainer_free(rt_dn_trainer* t) {
  for (void* a : t->allocs) cudaFree(a);
  t->allocs.clear();
  t->net.allocs.clear();  // the forward weights live in t->allocs
  delete t;
}

size_t buf_halves(const rt_dn_trainer* t, const DnOp& o) {
  return (size_t)t->planes * level_dim(t->H, o.level) * level_dim(t->W, o.level) * o.cout;
}
size_t align128(size_t n) { return (n + 127) & ~(size_t)127; }
}  // namespace

extern "C" {

rt_status rt_dn_train_create(rt_ctx* ctx, const void* blob, size_t bytes, uint32_t planes, uint32_t height,
                             uint32_t width, rt_dn_trainer** out) {
  if (!ctx || !blob || !out) return ctx_fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (planes == 0 || height == 0 || width == 0 || (uint64_t)planes * height * width > (1ull << 28))
    return ctx_fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad training batch shape");
  if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return ctx_fail(ctx, RT_ERR_CUDA, "cudaSetDevice");
  rt_dn_trainer* t = new rt_dn_trainer();
  t->ctx = ctx;
  t->planes = (int)planes;
  t->H = (int)height;
  t->W = (int)width;
  // parse with the inference loader (validates the op list), then keep the
  // blob's weights as FP32 masters
  std::string e = denoise_load(blob, bytes, &t->net);
  if (!e.empty()) {
    delete t;
    return ctx_fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  }
  if (!t->net.has_conf) {
    denoise_free(&t->net);
    delete t;
    return ctx_fail(ctx, RT_ERR_INVALID_ARGUMENT, "training needs a version 3 network (visibility and error outputs)");
  }
  // the loader's device copies are replaced by the trainer's own buffers
  for (void* a : t->net.allocs) cudaFree(a);
  t->net.allocs.clear();
  const unsigned char* p = static_cast<const unsigned char*>(blob);
  const uint32_t n_ops = t->net.ops.size();
  size_t off = 20 + 28 * (size_t)n_ops;  // version 3 header
  t->blob_head.assign(p, p + off);
  std::vector<float> host;
  for (const DnOp& o : t->net.ops) {
    t->conv_of_op.push_back(o.kind == DN_CONV ? (int)t->woff.size() : -1);
    if (o.kind != DN_CONV) continue;
    t->woff.push_back(host.size());
    const size_t nw = (size_t)o.cout * 9 * o.cin;
    for (size_t i = 0; i < nw; i++) {
      uint16_t h;
      memcpy(&h, p + off + 2 * i, 2);
      __half_raw r;
      r.x = h;
      host.push_back(__half2float(__half(r)));
    }
    off += 2 * nw;
    for (int i = 0; i < o.cout; i++) {
      float b;
      memcpy(&b, p + off + 4 * i, 4);
      host.push_back(b);
    }
    off += 4 * (size_t)o.cout;
  }
  t->n_params = (long long)host.size();
  auto bad = [&](const char* what) {
    trainer_free(t);
    return ctx_fail(ctx, RT_ERR_OUT_OF_MEMORY, std::string("training buffers: ") + what);
  };
  if (talloc(t, &t->master, host.size()) || talloc(t, &t->m1, host.size()) || talloc(t, &t->m2, host.size()) ||
      talloc(t, &t->grad, host.size()) || talloc(t, &t->acc, 4) || talloc(t, &t->zeros, 64) ||
      talloc(t, &t->err, 1))
    return bad("optimizer");
  cudaStream_t s = ctx_stream(ctx);
  if (cudaMemcpyAsync(t->master, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s) ||
      cudaMemsetAsync(t->m1, 0, host.size() * 4, s) || cudaMemsetAsync(t->m2, 0, host.size() * 4, s) ||
      cudaMemsetAsync(t->zeros, 0, 64 * 4, s))
    return bad("upload");
  for (size_t i = 0; i < t->net.ops.size(); i++) {
    DnOp& o = t->net.ops[i];
    if (o.kind != DN_CONV) continue;
    __half *fw, *bw;
    if (talloc(t, &fw, (size_t)o.cout * 9 * o.cin) || talloc(t, &bw, (size_t)o.cout * 9 * o.cin)) return bad("weights");
    o.w = fw;
    t->wbwd.push_back(bw);
    o.b = t->master + t->woff[t->conv_of_op[i]] + (size_t)o.cout * 9 * o.cin;
  }
  // activations (the inference arena: one buffer per op), their gradients,
  // the loss gradient and a temporary for backward data
  size_t na = 0, maxbuf = 0;
  t->act_off.assign(n_ops + 1, 0);
  for (size_t i = 0; i + 1 < n_ops; i++) {
    t->act_off[i + 1] = na;
    na = align128(na + buf_halves(t, t->net.ops[i]));
  }
  for (size_t i = 0; i < n_ops; i++) maxbuf = std::max(maxbuf, buf_halves(t, t->net.ops[i]));
  const size_t plane_px = (size_t)planes * height * width;
  maxbuf = std::max(maxbuf, plane_px * FEAT_CHANNELS);
  if (talloc(t, &t->arena, std::max(na, denoise_scratch_halves(t->net, t->planes, t->H, t->W))) ||
      talloc(t, &t->gbuf, std::max<size_t>(na, 128)) || talloc(t, &t->dz, maxbuf) ||
      talloc(t, &t->tmp, maxbuf) || talloc(t, &t->vis, plane_px * DN_MAX_SLOTS) ||
      talloc(t, &t->conf, plane_px * DN_MAX_SLOTS))
    return bad("activations");
  t->g_off = t->act_off;
  if (cudaStreamSynchronize(s) != cudaSuccess) return bad("sync");
  *out = t;
  return RT_OK;
}

void rt_dn_train_free(rt_dn_trainer* t) {
  if (!t) return;
  cudaSetDevice(ctx_device(t->ctx));
  cudaStreamSynchronize(ctx_stream(t->ctx));
  trainer_free(t);
}

}  // extern "C"

namespace {
// Forward + loss + backward of one batch; leaves the summed scaled gradient
// in t->grad and (count, visibility loss sum, error loss sum) in t->acc.
rt_status train_grads(rt_dn_trainer* t, const __half* feat, const __half* target, int* launches) {
  rt_ctx* ctx = t->ctx;
  cudaStream_t s = ctx_stream(ctx);
  const int nsm = ctx_num_sms(ctx);
  const int P = t->planes, H = t->H, W = t->W;
  const size_t nops = t->net.ops.size();
  auto CKE = [&](cudaError_t e, const char* what) -> bool {
    if (e == cudaSuccess) return true;
    ctx_fail(ctx, RT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
  };
  // FP16 operand layouts of the current masters
  for (size_t i = 0; i < nops; i++) {
    const DnOp& o = t->net.ops[i];
    if (o.kind != DN_CONV) continue;
    const long long n = (long long)o.cout * 9 * o.cin;
    k_pack_weights<<<grid_for(n, nsm), 256, 0, s>>>(t->master + t->woff[t->conv_of_op[i]], o.cin, o.cout,
                                                    (__half*)o.w, t->wbwd[t->conv_of_op[i]]);
    (*launches)++;
  }
  if (!CKE(cudaMemsetAsync(t->grad, 0, (size_t)t->n_params * 4, s), "memset") ||
      !CKE(cudaMemsetAsync(t->acc, 0, 4 * 4, s), "memset") || !CKE(cudaMemsetAsync(t->err, 0, 4, s), "memset"))
    return RT_ERR_CUDA;
  cudaError_t le = cudaSuccess;
  *launches += denoise_run(t->net, feat, P, H, W, t->arena, t->vis, t->conf, t->err, s, nsm, &le);
  if (!CKE(le, "forward")) return RT_ERR_CUDA;
  // activations by buffer id
  std::vector<const __half*> act(nops + 1, nullptr);
  act[0] = feat;
  for (size_t i = 0; i + 1 < nops; i++) act[i + 1] = t->arena + t->act_off[i + 1];
  auto G = [&](int b) { return t->gbuf + t->g_off[b]; };
  std::vector<bool> has(nops + 1, false);
  const long long npx = (long long)P * H * W;
  k_loss<<<grid_for(npx, nsm), 256, 0, s>>>(t->vis, t->conf, target, feat, t->dz, P, H, W, t->acc);
  (*launches)++;
  for (size_t ii = nops; ii-- > 0;) {
    const DnOp& o = t->net.ops[ii];
    const int b = (int)ii + 1;
    const int h = level_dim(H, o.level), w = level_dim(W, o.level);
    if (o.kind == DN_CONV) {
      const __half* dz = t->dz;
      if (ii + 1 < nops) {
        if (!has[b]) continue;  // nothing flows into this op's output
        const long long n8 = (long long)P * h * w * o.cout / 8;
        k_relu_mask<<<grid_for(n8, nsm), 256, 0, s>>>(G(b), act[b], t->dz, n8);
        (*launches)++;
      }
      const int c = t->conv_of_op[ii];
      float* dW = t->grad + t->woff[c];
      float* db = dW + (size_t)o.cout * 9 * o.cin;
      if (!CKE(wgrad_launch(o.cin, o.cout, act[o.src], dz, P, h, w, o.dil, dW, db, t->err, s, nsm), "wgrad"))
        return RT_ERR_CUDA;
      (*launches)++;
      if (o.src > 0) {
        // G[src] += transposed convolution of dZ (output: cin channels)
        if (!CKE(conv_launch(o.cout, o.cin, 3, dz, P, h, w, o.dil, t->wbwd[c], t->zeros, t->tmp, nullptr, nullptr,
                             nullptr, t->err, s, nsm),
                 "backward data"))
          return RT_ERR_CUDA;
        const long long n8 = (long long)P * h * w * o.cin / 8;
        k_acc<<<grid_for(n8, nsm), 256, 0, s>>>(G(o.src), t->tmp, n8, has[o.src] ? 0 : 1);
        *launches += 2;
        has[o.src] = true;
      }
    } else if (o.kind == DN_POOL) {
      if (!has[b]) continue;
      const int hi = level_dim(H, o.level - 1), wi = level_dim(W, o.level - 1);
      const long long n = (long long)P * hi * wi * o.cin / 8;
      k_pool_adj<<<grid_for(n, nsm), 256, 0, s>>>(G(b), G(o.src), P, hi, wi, o.cin, has[o.src] ? 0 : 1);
      (*launches)++;
      has[o.src] = true;
    } else {
      if (!has[b]) continue;
      const long long n8 = (long long)P * h * w * o.cin / 8;
      k_acc<<<grid_for(n8, nsm), 256, 0, s>>>(G(o.src2), G(b), n8, has[o.src2] ? 0 : 1);
      has[o.src2] = true;
      const int hl = level_dim(H, o.level + 1), wl = level_dim(W, o.level + 1);
      const long long nl = (long long)P * hl * wl * o.cin / 8;
      k_downsum<<<grid_for(nl, nsm), 256, 0, s>>>(G(b), G(o.src), P, h, w, o.cin, has[o.src] ? 0 : 1);
      *launches += 2;
      has[o.src] = true;
    }
  }
  // the loss gradient buffer dz is reused by the ReLU masks: the last op's
  // weight gradient reads it before the first mask overwrites it (reverse
  // order, one stream)
  if (!CKE(cudaGetLastError(), "launch")) return RT_ERR_CUDA;
  return RT_OK;
}
}  // namespace

extern "C" {

rt_status rt_dn_train_grads(rt_dn_trainer* t, const uint16_t* features, const uint16_t* targets, float* grads,
                            float* loss) {
  if (!t || !features || !targets) return ctx_fail(t ? t->ctx : nullptr, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (((uintptr_t)features & 15) != 0)
    return ctx_fail(t->ctx, RT_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
  cudaSetDevice(ctx_device(t->ctx));
  int launches = 0;
  rt_status st = train_grads(t, reinterpret_cast<const __half*>(features), reinterpret_cast<const __half*>(targets),
                             &launches);
  if (st != RT_OK) return st;
  cudaStream_t s = ctx_stream(t->ctx);
  float hacc[4];
  int herr = 0;
  if (grads) cudaMemcpyAsync(grads, t->grad, (size_t)t->n_params * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hacc, t->acc, sizeof hacc, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&herr, t->err, 4, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return ctx_fail(t->ctx, RT_ERR_CUDA, std::string("training step: ") + cudaGetErrorString(e));
  if (herr & DN_ERR_WAIT) return ctx_fail(t->ctx, RT_ERR_DEVICE_WATCHDOG, "training: a tensor-core wait timed out");
  if (loss) {
    loss[0] = hacc[0];
    loss[1] = hacc[1];
    loss[2] = hacc[2];
  }
  if (grads) {
    // unscale: the gradient of the summed (not averaged) loss
    for (long long i = 0; i < t->n_params; i++) grads[i] /= kLossScale;
  }
  return RT_OK;
}

rt_status rt_dn_train_step(rt_dn_trainer* t, const uint16_t* features, const uint16_t* targets, float lr, float beta1,
                           float beta2, float eps, float* loss) {
  if (!t || !features || !targets) return ctx_fail(t ? t->ctx : nullptr, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (((uintptr_t)features & 15) != 0)
    return ctx_fail(t->ctx, RT_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
  cudaSetDevice(ctx_device(t->ctx));
  int launches = 0;
  rt_status st = train_grads(t, reinterpret_cast<const __half*>(features), reinterpret_cast<const __half*>(targets),
                             &launches);
  if (st != RT_OK) return st;
  cudaStream_t s = ctx_stream(t->ctx);
  t->steps++;
  const float bc1 = 1.f - std::pow(beta1, (float)t->steps), bc2 = 1.f - std::pow(beta2, (float)t->steps);
  k_grad_check<<<grid_for(t->n_params, ctx_num_sms(t->ctx)), 256, 0, s>>>(t->grad, t->n_params, t->acc);
  k_adam<<<grid_for(t->n_params, ctx_num_sms(t->ctx)), 256, 0, s>>>(t->master, t->m1, t->m2, t->grad, t->n_params,
                                                                     t->acc, lr, beta1, beta2, eps, bc1, bc2);
  if (loss) {
    float hacc[4];
    int herr = 0;
    cudaMemcpyAsync(hacc, t->acc, sizeof hacc, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&herr, t->err, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
      return ctx_fail(t->ctx, RT_ERR_CUDA, std::string("training step: ") + cudaGetErrorString(e));
    if (herr & DN_ERR_WAIT) return ctx_fail(t->ctx, RT_ERR_DEVICE_WATCHDOG, "training: a tensor-core wait timed out");
    loss[0] = hacc[0];
    loss[1] = hacc[1];
    loss[2] = hacc[2];
    loss[3] = hacc[3];
  } else if (cudaGetLastError() != cudaSuccess) {
    return ctx_fail(t->ctx, RT_ERR_CUDA, "training step launch failed");
  }
  return RT_OK;
}

rt_status rt_dn_train_export(rt_dn_trainer* t, void* blob_out, size_t* bytes) {
  if (!t || !bytes) return ctx_fail(t ? t->ctx : nullptr, RT_ERR_INVALID_ARGUMENT, "null argument");
  size_t need = t->blob_head.size();
  for (const DnOp& o : t->net.ops)
    if (o.kind == DN_CONV) need += (size_t)o.cout * 9 * o.cin * 2 + (size_t)o.cout * 4;
  if (!blob_out) {
    *bytes = need;
    return RT_OK;
  }
  if (*bytes < need) return ctx_fail(t->ctx, RT_ERR_INVALID_ARGUMENT, "export buffer too small");
  std::vector<float> host((size_t)t->n_params);
  cudaSetDevice(ctx_device(t->ctx));
  cudaStream_t s = ctx_stream(t->ctx);
  cudaMemcpyAsync(host.data(), t->master, host.size() * 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return ctx_fail(t->ctx, RT_ERR_CUDA, "export: copy failed");
  unsigned char* o = static_cast<unsigned char*>(blob_out);
  memcpy(o, t->blob_head.data(), t->blob_head.size());
  size_t off = t->blob_head.size();
  for (size_t i = 0; i < t->net.ops.size(); i++) {
    const DnOp& op = t->net.ops[i];
    if (op.kind != DN_CONV) continue;
    const size_t w0 = t->woff[t->conv_of_op[i]], nw = (size_t)op.cout * 9 * op.cin;
    for (size_t k = 0; k < nw; k++) {
      __half h = __float2half_rn(host[w0 + k]);
      memcpy(o + off + 2 * k, &h, 2);
    }
    off += 2 * nw;
    memcpy(o + off, host.data() + w0 + nw, (size_t)op.cout * 4);
    off += (size_t)op.cout * 4;
  }
  *bytes = need;
  return RT_OK;
}

rt_status rt_dn_train_set_threshold(rt_dn_trainer* t, float threshold) {
  if (!t || !(threshold >= 0.0f)) return ctx_fail(t ? t->ctx : nullptr, RT_ERR_INVALID_ARGUMENT, "bad threshold");
  memcpy(t->blob_head.data() + 16, &threshold, 4);
  return RT_OK;
}

rt_status rt_debug_conv_wgrad(rt_ctx* ctx, const uint16_t* x, const uint16_t* dz, uint32_t planes, uint32_t height,
                              uint32_t width, uint32_t cin, uint32_t cout, uint32_t dil, float* dw, float* db) {
  if (!ctx || !x || !dz || !dw || !db) return ctx_fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  cudaSetDevice(ctx_device(ctx));
  cudaStream_t s = ctx_stream(ctx);
  int* err = nullptr;
  if (cudaMalloc((void**)&err, 4) != cudaSuccess) return ctx_fail(ctx, RT_ERR_OUT_OF_MEMORY, "cudaMalloc");
  cudaMemsetAsync(err, 0, 4, s);
  cudaError_t e = wgrad_launch((int)cin, (int)cout, reinterpret_cast<const __half*>(x),
                               reinterpret_cast<const __half*>(dz), (int)planes, (int)height, (int)width, (int)dil, dw,
                               db, err, s, ctx_num_sms(ctx));
  int herr = 0;
  if (e == cudaSuccess) {
    cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
  }
  cudaFree(err);
  if (e != cudaSuccess) return ctx_fail(ctx, RT_ERR_CUDA, std::string("wgrad: ") + cudaGetErrorString(e));
  if (herr & DN_ERR_WAIT) return ctx_fail(ctx, RT_ERR_DEVICE_WATCHDOG, "wgrad: a tensor-core wait timed out");
  return RT_OK;
}

}  // extern "C"
