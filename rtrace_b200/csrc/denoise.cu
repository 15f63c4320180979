// Dilated 3x3 convolutions of the soft-shadow denoiser on the 5th-generation
// tensor cores.
//
// One CTA of 128 threads owns a 128-pixel run of one image row (the GEMM's
// M = 128) and computes all output channels (N = COUT) over K = 9 * CIN
// (nine taps times the input channels):
//   1. the nine shifted input runs are staged in shared memory in the
//      tcgen05 K-major, no-swizzle operand layout: 8-row x 16-byte core
//      matrices, one 2 KB block per 8 input channels of a tap (rows 16 bytes
//      apart, blocks 2 KB apart); out-of-image taps are zero-filled;
//   2. one thread issues K / 16 tcgen05.mma (kind::f16, FP32 accumulate)
//      into a TMEM accumulator of COUT columns and commits them to an
//      mbarrier;
//   3. each warp reads its 32 accumulator lanes (tcgen05.ld 32x32b), adds
//      the bias, applies the activation and stores FP16 (or, for the last
//      layer, the sigmoid visibility as float).
// The weights (K x COUT, same layout) stay in shared memory for the CTA's
// whole persistent loop.  Every wait is bounded; a wait that runs out sets
// the error word and the CTA leaves after releasing its tensor memory.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "denoise.hpp"

namespace rtb {
namespace {

constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading byte offset (between the two 8-element K halves of one MMA step),
// stride byte offset (between 8-row groups), version 1 for sm_100.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, FP16 A and B, both
// K-major, M and N encoded as M >> 4 and N >> 3.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
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

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[N]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

constexpr int TILE_M = 128;
constexpr int TMEM_COLS = 32;  // >= COUT, power of two >= 32

template <int CIN, int COUT>
struct ConvSmem {
  static constexpr int KCH = 9 * CIN / 8;                 // 16-byte K chunks
  static constexpr int A_BYTES = KCH * TILE_M * 16;       // im2col tile
  static constexpr int B_BYTES = KCH * COUT * 16;         // weights
  // 32 KB of slack past the operands: a descriptor whose strides were
  // misread would still read inside the CTA's own shared memory
  static constexpr int SLACK = 32 * 1024;
  static constexpr int TOTAL = 1024 + A_BYTES + B_BYTES + 64 + SLACK;
};

// MODE 0: ReLU, FP16 output [plane][H][W][COUT].  MODE 2: sigmoid of the
// first DN_MAX_SLOTS channels, float output [plane][slot][H][W].
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(128) k_conv3x3_tc(const __half* __restrict__ in, int planes, int H, int W, int dil,
                                                     const uint4* __restrict__ wl, const float* __restrict__ bias,
                                                     __half* __restrict__ out, float* __restrict__ vis, int* err) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= TMEM_COLS, "unsupported channel counts");
  using SM = ConvSmem<CIN, COUT>;
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte aligned operand region
  uint32_t raw = smem_u32(smem_raw);
  uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* base = smem_raw + pad;
  const uint32_t sA = raw + pad;
  const uint32_t sB = sA + SM::A_BYTES;
  unsigned char* tail = base + SM::A_BYTES + SM::B_BYTES;
  uint64_t* mbar_p = reinterpret_cast<uint64_t*>(tail);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tail + 8);
  volatile int* s_fail = reinterpret_cast<volatile int*>(tail + 16);
  const uint32_t mbar = smem_u32(mbar_p);
  const int tid = threadIdx.x, warp = tid >> 5;

  // weights -> shared memory (already in operand layout)
  {
    uint4* dst = reinterpret_cast<uint4*>(base + SM::A_BYTES);
    for (int i = tid; i < SM::B_BYTES / 16; i += 128) dst[i] = wl[i];
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t IDESC = umma_idesc(TILE_M, COUT);
  constexpr int KSTEPS = 9 * CIN / 16;
  constexpr int CPT = CIN / 8;  // chunks per tap

  const int tiles_x = (W + TILE_M - 1) / TILE_M;
  const long long ntiles = (long long)planes * H * tiles_x;
  uint32_t phase = 0;
  bool failed = false;
  for (long long tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const int tx = (int)(tile % tiles_x);
    const long long py = tile / tiles_x;
    const int y = (int)(py % H);
    const long long p = py / H;
    const int x0 = tx * TILE_M;
    // 1. im2col: q -> (tap, pixel, chunk), chunk fastest so that a warp reads
    // consecutive 16-byte pieces of consecutive pixels
    for (int q = tid; q < 9 * TILE_M * CPT; q += 128) {
      const int j = q % CPT;
      const int rest = q / CPT;
      const int r = rest % TILE_M;
      const int t = rest / TILE_M;
      const int xs = x0 + r + (t % 3 - 1) * dil;
      const int ys = y + (t / 3 - 1) * dil;
      const bool ok = xs >= 0 && xs < W && ys >= 0 && ys < H;
      const __half* src = ok ? in + ((p * H + ys) * (long long)W + xs) * CIN + 8 * j : in;
      cp_async16(sA + (uint32_t)((t * CPT + j) * (TILE_M * 16) + r * 16), src, ok ? 16 : 0);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // 2. the MMA chain, issued by one thread
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < KSTEPS; s++) {
        uint64_t da = umma_desc(sA + (uint32_t)(s * 2 * TILE_M * 16), TILE_M * 16, 128);
        uint64_t db = umma_desc(sB + (uint32_t)(s * 2 * COUT * 16), COUT * 16, 128);
        mma_f16(tmem, da, db, IDESC, s > 0 ? 1u : 0u);
      }
      mma_commit(mbar);
    }
    // thread 0 waits for the chain (bounded) and publishes the outcome, so
    // that every thread takes the same path below
    if (tid == 0) {
      int f = 0;
      if (!mbar_wait(mbar, phase)) {
        atomicOr(err, DN_ERR_WAIT);
        f = 1;
        mbar_wait(mbar, phase);  // give the chain a second bound before TMEM is released
      }
      *s_fail = f;
    }
    __syncthreads();
    if (*s_fail) {
      failed = true;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // 3. epilogue: thread tid owns accumulator row (pixel) tid
    uint32_t acc[COUT];
    tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16), acc);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int x = x0 + tid;
    if (x < W) {
      if (MODE == 0) {
        __half* o = out + ((p * H + y) * (long long)W + x) * COUT;
#pragma unroll
        for (int c = 0; c < COUT; c += 8) {
          __align__(16) __half h[8];
#pragma unroll
          for (int e = 0; e < 8; e++) {
            float v = __uint_as_float(acc[c + e]) + __ldg(bias + c + e);
            h[e] = __float2half_rn(v > 0.f ? v : 0.f);
          }
          *reinterpret_cast<uint4*>(o + c) = *reinterpret_cast<const uint4*>(h);
        }
      } else {
#pragma unroll
        for (int j = 0; j < DN_MAX_SLOTS; j++) {
          float v = __uint_as_float(acc[j]) + __ldg(bias + j);
          vis[((p * DN_MAX_SLOTS + j) * H + y) * (long long)W + x] = 1.f / (1.f + __expf(-v));
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

template <int CIN, int COUT, int MODE>
cudaError_t launch_conv(const __half* in, int planes, int H, int W, int dil, const void* w, const float* b, __half* out,
                        float* vis, int* err, cudaStream_t s, int num_sms) {
  using SM = ConvSmem<CIN, COUT>;
  static unsigned long long attr_set = 0;  // one bit per device ordinal (< 64)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  unsigned long long bit = dev < 64 ? 1ull << dev : 0;
  if (!(attr_set & bit)) {
    e = cudaFuncSetAttribute(k_conv3x3_tc<CIN, COUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::TOTAL);
    if (e != cudaSuccess) return e;
    attr_set |= bit;
  }
  long long ntiles = (long long)planes * H * ((W + TILE_M - 1) / TILE_M);
  long long grid = std::min<long long>(ntiles, (long long)num_sms * 2);
  if (grid < 1) grid = 1;
  k_conv3x3_tc<CIN, COUT, MODE><<<(int)grid, 128, SM::TOTAL, s>>>(in, planes, H, W, dil, (const uint4*)w, b, out, vis,
                                                                  err);
  return cudaGetLastError();
}

float half_to_float_host(uint16_t h) {
  __half_raw r;
  r.x = h;
  return __half2float(__half(r));
}

}  // namespace

std::string denoise_load(const void* blob, size_t bytes, DenoiseNet* net) {
  denoise_free(net);
  const unsigned char* p = static_cast<const unsigned char*>(blob);
  auto u32 = [&](size_t off) {
    uint32_t v;
    memcpy(&v, p + off, 4);
    return v;
  };
  if (!blob || bytes < 12 || memcmp(p, "RTDN", 4) != 0) return "not a denoiser weight blob (magic RTDN)";
  if (u32(4) != 1) return "unsupported denoiser blob version";
  uint32_t n = u32(8);
  if (n < 1 || n > 32) return "denoiser layer count must be 1..32";
  size_t off = 12 + 16 * (size_t)n;
  if (bytes < off) return "truncated denoiser blob";
  std::vector<DnLayer> L(n);
  for (uint32_t i = 0; i < n; i++) {
    L[i].cin = (int)u32(12 + 16 * i);
    L[i].cout = (int)u32(16 + 16 * i);
    L[i].dil = (int)u32(20 + 16 * i);
    L[i].act = (int)u32(24 + 16 * i);
    bool last = i + 1 == n;
    if ((L[i].cin != 16 && L[i].cin != 32) || (L[i].cout != 16 && L[i].cout != 32))
      return "denoiser layers must have 16 or 32 input and output channels";
    if (L[i].dil < 1 || L[i].dil > 256) return "denoiser dilation must be 1..256";
    if (L[i].act != (last ? 2 : 0)) return "denoiser layers must be ReLU, the last one sigmoid";
    if (last && L[i].cout != 16) return "the last denoiser layer must have 16 output channels";
    if (i == 0 && L[i].cin != FEAT_CHANNELS) return "the first denoiser layer must read 16 feature channels";
    if (i > 0 && L[i].cin != L[i - 1].cout) return "denoiser layer channel counts do not chain";
  }
  std::vector<void*> allocs;
  auto fail = [&](const std::string& m) {
    for (void* a : allocs) cudaFree(a);
    return m;
  };
  size_t params = 0;
  for (uint32_t i = 0; i < n; i++) {
    const int cin = L[i].cin, cout = L[i].cout, K = 9 * cin;
    size_t wbytes = (size_t)cout * K * 2, bbytes = (size_t)cout * 4;
    if (bytes < off + wbytes + bbytes) return fail("truncated denoiser blob");
    const uint16_t* w = reinterpret_cast<const uint16_t*>(p + off);
    // [cout][ky][kx][cin] -> operand layout: K chunk k/8 at k/8 * (cout*16),
    // row n at n * 16, element k%8 at 2 * (k%8); k = (ky*3 + kx) * cin + c
    std::vector<uint16_t> lay((size_t)cout * K, 0);
    for (int nn = 0; nn < cout; nn++)
      for (int k = 0; k < K; k++) {
        uint16_t v;
        memcpy(&v, w + (size_t)nn * K + k, 2);
        size_t dst = ((size_t)(k / 8) * (cout * 16) + (size_t)nn * 16 + (size_t)(k % 8) * 2) / 2;
        lay[dst] = v;
        if (half_to_float_host(v) != half_to_float_host(v)) return fail("NaN in denoiser weights");
      }
    void* dw = nullptr;
    float* db = nullptr;
    if (cudaMalloc(&dw, wbytes) != cudaSuccess) return fail("cudaMalloc(denoiser weights) failed");
    allocs.push_back(dw);
    if (cudaMalloc((void**)&db, bbytes) != cudaSuccess) return fail("cudaMalloc(denoiser bias) failed");
    allocs.push_back(db);
    if (cudaMemcpy(dw, lay.data(), wbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db, p + off + wbytes, bbytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail("uploading denoiser weights failed");
    L[i].w = dw;
    L[i].b = db;
    off += wbytes + bbytes;
    params += (size_t)cout * K + cout;
  }
  if (off != bytes) return fail("denoiser blob has trailing bytes");
  net->layers = L;
  net->allocs = allocs;
  net->param_count = params;
  return std::string();
}

void denoise_free(DenoiseNet* net) {
  for (void* a : net->allocs) cudaFree(a);
  net->allocs.clear();
  net->layers.clear();
  net->param_count = 0;
}

int denoise_run(const DenoiseNet& net, const __half* feat, int planes, int H, int W, __half* act0, __half* act1,
                float* vis, int* err, cudaStream_t s, int num_sms, cudaError_t* launch_err) {
  const __half* cur = feat;
  int launches = 0;
  *launch_err = cudaSuccess;
  for (size_t i = 0; i < net.layers.size(); i++) {
    const DnLayer& l = net.layers[i];
    __half* out = (i % 2 == 0) ? act0 : act1;
    cudaError_t e = cudaErrorInvalidValue;
    if (l.act == 2) {
      if (l.cin == 16) e = launch_conv<16, 16, 2>(cur, planes, H, W, l.dil, l.w, l.b, nullptr, vis, err, s, num_sms);
      else e = launch_conv<32, 16, 2>(cur, planes, H, W, l.dil, l.w, l.b, nullptr, vis, err, s, num_sms);
    } else if (l.cin == 16 && l.cout == 16) {
      e = launch_conv<16, 16, 0>(cur, planes, H, W, l.dil, l.w, l.b, out, nullptr, err, s, num_sms);
    } else if (l.cin == 16 && l.cout == 32) {
      e = launch_conv<16, 32, 0>(cur, planes, H, W, l.dil, l.w, l.b, out, nullptr, err, s, num_sms);
    } else if (l.cin == 32 && l.cout == 16) {
      e = launch_conv<32, 16, 0>(cur, planes, H, W, l.dil, l.w, l.b, out, nullptr, err, s, num_sms);
    } else {
      e = launch_conv<32, 32, 0>(cur, planes, H, W, l.dil, l.w, l.b, out, nullptr, err, s, num_sms);
    }
    launches++;
    if (e != cudaSuccess) {
      *launch_err = e;
      return launches;
    }
    cur = out;
  }
  return launches;
}

}  // namespace rtb
