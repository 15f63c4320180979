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

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

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
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, uint32_t (&r)[32]);

template <>
__device__ __forceinline__ void tmem_ld<64>(uint32_t taddr, uint32_t (&r)[64]) {
  tmem_ld<32>(taddr, *reinterpret_cast<uint32_t(*)[32]>(&r[0]));
  tmem_ld<32>(taddr + 32u, *reinterpret_cast<uint32_t(*)[32]>(&r[32]));
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
constexpr int MAX_DIL = 64;    // 128 + 2 * dilation pixels must fit one TMA box (<= 256)
// TMEM columns of one accumulator (>= COUT, at least 32) and of a CTA's
// allocation (NACC accumulators, a power of two >= 32)
__host__ __device__ constexpr int acc_cols(int cout) { return cout < 32 ? 32 : cout; }

// Shared memory of one CTA: a ring of NROW staged input rows (TILE_M +
// 2 * dil pixels each, one block of 16-byte rows per 8 channels), the
// weights, the pipeline's mbarriers, the TMEM address and an abort flag.
// A step reads 3 rows, so the TMA warp runs NROW - 3 rows ahead.  Fewer
// rows let more CTAs share an SM, which hides more than deeper prefetch
// does (measured on the network at 1080p x 4: 4 rows everywhere 2.68 ms,
// 6 everywhere 2.87 ms, 6 for the 64-channel shapes 2.71 ms); 64 -> 32 fits
// two CTAs per SM only with 3 rows (2.62 ms).
__host__ __device__ constexpr int conv_nrow(int cin, int cout) { return (cin == 64 && cout == 32) ? 3 : 4; }
constexpr int NACC = 2;    // TMEM accumulators (MMA -> epilogue)
constexpr int SEG = 8;     // output rows a CTA walks down one column at a time (8 measured best of 8-64)
constexpr int CONV_THREADS = 192;  // warps 0-3 epilogue, warp 4 TMA, warp 5 MMA
// Register cap: the pooling epilogue (MODE 4) of 32 -> 32 keeps 32 running
// sums per thread; without a cap it takes 128 registers and 2 CTAs per SM
// where shared memory allows 3.
__host__ __device__ constexpr int conv_min_blocks(int cin, int cout, int mode) {
  return (mode == 4 && cin == 32 && cout == 32) ? 3 : 1;
}
__host__ __device__ constexpr int halo_px(int dil) { return TILE_M + 2 * dil; }
__host__ __device__ constexpr int halo_block(int dil) { return ((halo_px(dil) * 16 + 127) / 128) * 128; }
template <int CIN, int COUT>
struct ConvSmem {
  static constexpr int NROW = conv_nrow(CIN, COUT);       // staged input rows (TMA -> MMA)
  static constexpr int CPT = CIN / 8;                     // 16-byte channel chunks per pixel
  static constexpr int B_BYTES = 9 * CPT * COUT * 16;     // weights
  static constexpr int TAIL = 256;                        // barriers, TMEM slot, abort flag
  static_assert(8 * (2 * NROW + 2 * NACC) + 8 <= TAIL, "the mbarriers, TMEM slot and abort flag overflow TAIL");
  static constexpr int BIAS = 256;                        // COUT floats
  static constexpr int OUT = 4 * 32 * COUT * 2;           // epilogue staging: 32 pixels per warp
  static int row_bytes(int dil) { return CPT * halo_block(dil); }
  static int total(int dil) { return 1024 + NROW * row_bytes(dil) + B_BYTES + TAIL + BIAS + OUT; }
};

// Work of the convolution: segments of up to SEG output rows of one column
// (plane p, 128-pixel tile tx, rows y = r, r + dil, r + 2 dil, ... of one
// residue r mod dil).  Output row y reads input rows y - dil, y, y + dil,
// so consecutive rows of a column share two of their three input rows: a
// segment of L rows stages L + 2 input rows instead of 3L.
struct ConvSeg {
  int p, tx, r, k0, L;  // rows y = r + (k0 + t) * dil for t < L
};
__device__ __forceinline__ int conv_col_segs(int H, int dil) { return ((H + dil - 1) / dil + SEG - 1) / SEG; }
__device__ __forceinline__ ConvSeg conv_seg(long long g, int H, int dil, int tiles_x) {
  const int nseg = conv_col_segs(H, dil);
  ConvSeg c;
  const int q = (int)(g % nseg);
  long long col = g / nseg;
  c.r = (int)(col % dil);
  col /= dil;
  c.tx = (int)(col % tiles_x);
  c.p = (int)(col / tiles_x);
  c.k0 = q * SEG;
  const int rows = (H - c.r + dil - 1) / dil;  // rows of residue r below H
  c.L = max(0, min(SEG, rows - c.k0));
  return c;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// Epilogue modes.  FP16 NHWC output [plane][H][W][COUT]:
//   MODE 0: bias + ReLU (forward hidden layers);
//   MODE 1: the accumulator times (aux > 0), aux an FP16 NHWC tensor of the
//           output's shape, no bias (backward data through a ReLU: aux is
//           the forward activation the gradient flows into);
//   MODE 3: the accumulator alone (backward data into a linear tensor);
//   MODE 4: MODE 0, and the output's 2x2 average pool (k_pool2's bytes)
//           into `pool`, for a layer of dilation 1 that a pooling follows.
// MODE 2: float outputs: sigmoid(channel j + bias) for j < DN_MAX_SLOTS
// into vis [plane][slot][H][W] (visibility of disk-light slot j) and
// sigmoid(channel DN_MAX_SLOTS + j + bias) into conf (the network's
// estimate of its own error on slot j), if conf is not null.
//
// A step is one 128-pixel run of one output row; the CTA walks segments
// blockIdx.x, blockIdx.x + gridDim.x, ... (see ConvSeg), a segment's steps
// down its column, with three roles working on different steps:
//   warp 4 (TMA): loads input row j (count over the CTA's whole walk) into
//     ring slot j % NROW with CIN / 8 boxes (8 channels x halo_px pixels of
//     one row; the hardware zero-fills outside the image and the plane),
//     once the MMAs of row j - NROW's last step have released the slot;
//   warp 5 (MMA): for step t of a segment whose first row is j0, once rows
//     j0 + t .. j0 + t + 2 have landed and the epilogue has drained
//     accumulator i % NACC, issues the 9 * CIN / 16 MMAs; tap (ky, kx) reads
//     row j0 + t + ky's slot from pixel kx * dil on (descriptor start
//     kx * dil * 16 bytes further); commits to the accumulator's "full"
//     barrier and to the "empty" barrier of row j0 + t (and, at a
//     segment's last step, of its last two rows), each row's last use;
//   warps 0-3 (epilogue): thread t reads accumulator row t (tcgen05.ld
//     32x32b), releases the accumulator, adds the bias, applies the
//     activation and stores.
// Every wait is bounded; one that runs out raises the abort flag, all roles
// leave their loops, and the TMA and MMA threads wait (bounded) for their
// operations still in flight before the tensor memory is released.
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(CONV_THREADS, conv_min_blocks(CIN, COUT, MODE)) k_conv3x3_tc(const __grid_constant__ CUtensorMap in_map, int planes,
                                                              int H, int W, int dil, const uint4* __restrict__ wl,
                                                              const float* __restrict__ bias,
                                                              __half* __restrict__ out, float* __restrict__ vis,
                                                              float* __restrict__ conf,
                                                              const __half* __restrict__ aux,
                                                              __half* __restrict__ pool, int* err) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 64, "unsupported channel counts");
  constexpr int ACC = acc_cols(COUT), TMEM_ALLOC = NACC * ACC;
  using SM = ConvSmem<CIN, COUT>;
  constexpr int CPT = SM::CPT;
  constexpr int NROW = SM::NROW;
  extern __shared__ unsigned char smem_raw[];
  uint32_t raw = smem_u32(smem_raw);
  uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* base = smem_raw + pad;
  const int BLK = halo_block(dil);
  const int ROWB = CPT * BLK;
  const uint32_t sA = raw + pad;  // ring slot k at sA + k * ROWB
  const uint32_t sB = sA + NROW * ROWB;
  unsigned char* tail = base + NROW * ROWB + SM::B_BYTES;
  const uint32_t bar0 = smem_u32(tail);  // full[NROW], empty[NROW], accf[NACC], acce[NACC]
  auto full_bar = [&](int k) { return bar0 + 8u * k; };
  auto empty_bar = [&](int k) { return bar0 + 8u * (NROW + k); };
  auto accf_bar = [&](int k) { return bar0 + 8u * (2 * NROW + k); };
  auto acce_bar = [&](int k) { return bar0 + 8u * (2 * NROW + NACC + k); };
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tail + 8 * (2 * NROW + 2 * NACC));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tail + 8 * (2 * NROW + 2 * NACC) + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  float* s_bias = reinterpret_cast<float*>(tail + SM::TAIL);
  unsigned char* s_out = tail + SM::TAIL + SM::BIAS;  // 4 warps x 32 pixels x COUT halves
  {
    uint4* dst = reinterpret_cast<uint4*>(base + NROW * ROWB);
    for (int i = tid; i < SM::B_BYTES / 16; i += CONV_THREADS) dst[i] = wl[i];
    for (int i = tid; i < COUT; i += CONV_THREADS) s_bias[i] = bias[i];
  }
  if (tid == 0) {
    for (int k = 0; k < NROW; k++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full_bar(k)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty_bar(k)) : "memory");
    }
    for (int k = 0; k < NACC; k++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(accf_bar(k)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(acce_bar(k)) : "memory");
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&in_map)) : "memory");
  }
  if (warp == 5) {
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_ALLOC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t IDESC = umma_idesc(TILE_M, COUT);
  const uint32_t tx_bytes = (uint32_t)(CPT * halo_px(dil) * 16);  // one staged row
  const int tiles_x = (W + TILE_M - 1) / TILE_M;
  const long long nsegs = (long long)planes * tiles_x * dil * conv_col_segs(H, dil);
  auto fail = [&]() {
    if (!*abort_flag) atomicOr(err, DN_ERR_WAIT);
    *abort_flag = 1;
  };

  if (warp == 4) {
    // ---- TMA producer: the rows of each segment, r + (k0 - 1 + j) * dil
    if (lane == 0) {
      long long issued = 0;
      bool stop = false;
      for (long long g = blockIdx.x; g < nsegs && !stop; g += gridDim.x) {
        const ConvSeg c = conv_seg(g, H, dil, tiles_x);
        for (int j = 0; j < (c.L > 0 ? c.L + 2 : 0); j++, issued++) {
          const int k = (int)(issued % NROW);
          if (*abort_flag || !mbar_wait(empty_bar(k), (uint32_t)((issued / NROW) & 1) ^ 1u)) {
            fail();
            stop = true;
            break;
          }
          mbar_expect_tx(full_bar(k), tx_bytes);
          const uint32_t st = sA + (uint32_t)(k * ROWB);
          const int y = c.r + (c.k0 - 1 + j) * dil;
          for (int cc = 0; cc < CPT; cc++)
            tma_load_4d(st + (uint32_t)(cc * BLK), &in_map, 8 * cc, c.tx * TILE_M - dil, y, c.p, full_bar(k));
        }
      }
      if (*abort_flag) {
        // let the last loads land before the CTA's shared memory goes away
        for (long long k = issued - NROW; k < issued; k++)
          if (k >= 0) mbar_wait(full_bar((int)(k % NROW)), (uint32_t)((k / NROW) & 1));
      }
    }
  } else if (warp == 5) {
    // ---- MMA issuer
    if (lane == 0) {
      long long i = 0, j0 = 0;  // steps issued; the segment's first row
      bool stop = false;
      for (long long g = blockIdx.x; g < nsegs && !stop; g += gridDim.x) {
        const ConvSeg c = conv_seg(g, H, dil, tiles_x);
        if (c.L <= 0) continue;
        for (int t = 0; t < c.L; t++, i++) {
          const int a = (int)(i % NACC);
          bool ok = !*abort_flag;
          for (int ky = 0; ky < 3 && ok; ky++) {
            const long long j = j0 + t + ky;
            ok = mbar_wait(full_bar((int)(j % NROW)), (uint32_t)((j / NROW) & 1));
          }
          if (!ok || !mbar_wait(acce_bar(a), (uint32_t)((i / NACC) & 1) ^ 1u)) {
            fail();
            stop = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t acc = tmem + (uint32_t)(a * ACC);
#pragma unroll
          for (int tap = 0; tap < 9; tap++) {
            const int ky = tap / 3, kx = tap % 3;
            const uint32_t row = sA + (uint32_t)(((j0 + t + ky) % NROW) * ROWB);
#pragma unroll
            for (int s2 = 0; s2 < CIN / 16; s2++) {
              uint64_t da = umma_desc(row + (uint32_t)(2 * s2 * BLK + kx * dil * 16), (uint32_t)BLK, 128);
              uint64_t db = umma_desc(sB + (uint32_t)((tap * CPT + 2 * s2) * COUT * 16), COUT * 16, 128);
              mma_f16(acc, da, db, IDESC, (tap > 0 || s2 > 0) ? 1u : 0u);
            }
          }
          mma_commit(empty_bar((int)((j0 + t) % NROW)));
          if (t == c.L - 1) {
            mma_commit(empty_bar((int)((j0 + t + 1) % NROW)));
            mma_commit(empty_bar((int)((j0 + t + 2) % NROW)));
          }
          mma_commit(accf_bar(a));
        }
        j0 += c.L + 2;
      }
      if (*abort_flag && i > 0) mbar_wait(accf_bar((int)((i - 1) % NACC)), (uint32_t)(((i - 1) / NACC) & 1));
    }
  } else {
    // ---- epilogue (warps 0-3: thread tid <-> TMEM lane tid <-> pixel x0 + tid)
    long long i = 0;
    bool stop = false;
    // MODE 4: the running 2x2 sums of the pooled pixel this lane (even
    // lanes: pixels x, x + 1; rows y, y + 1 are consecutive steps of a
    // segment) writes, added in k_pool2's order
    float pacc[MODE == 4 ? COUT : 1];
    for (long long g = blockIdx.x; g < nsegs && !stop; g += gridDim.x) {
      const ConvSeg c = conv_seg(g, H, dil, tiles_x);
      for (int t = 0; t < c.L; t++, i++) {
        const int a = (int)(i % NACC);
        bool ok = true;
        for (long long k = 0; k < kWaitLimit; k++) {
          uint32_t done;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
              "selp.u32 %0, 1, 0, p;\n\t"
              "}\n"
              : "=r"(done)
              : "r"(accf_bar(a)), "r"((uint32_t)((i / NACC) & 1))
              : "memory");
          if (done) break;
          if (*abort_flag || k + 1 == kWaitLimit) {
            ok = false;
            break;
          }
        }
        // the four warps agree before the warp-collective TMEM load
        if (__any_sync(0xffffffffu, !ok)) ok = false;
        if (!ok) {
          if (lane == 0) fail();
          stop = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t accv[COUT];
        tmem_ld<COUT>(tmem + (uint32_t)(a * ACC) + ((uint32_t)(warp * 32) << 16), accv);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if (lane == 0) mbar_arrive(acce_bar(a));
        const int tx = c.tx, p = c.p, y = c.r + (c.k0 + t) * dil;
        const int x = tx * TILE_M + tid;
        // MODE 4 (dilation 1, segments start on even rows): rows y, y + 1 of
        // a pooled row are steps t, t + 1; an odd count ends at the image's
        // last row
        const bool odd_row = (t & 1) != 0, pool_row = odd_row || t + 1 == c.L, pair_x = x + 1 < W;
        if (MODE != 2) {
          constexpr int CPX0 = COUT / 8;
          // MODE 1: the ReLU mask of this pixel's forward activation
          uint4 mk[CPX0];
          if (MODE == 1 && x < W) {
            const uint4* ap = reinterpret_cast<const uint4*>(aux + (((long long)p * H + y) * (long long)W + x) * COUT);
  #pragma unroll
            for (int c = 0; c < CPX0; c++) mk[c] = ap[c];
          }
          // Each warp stages its 32 pixels (COUT halves each) in shared
          // memory, 16-byte chunks XOR-swizzled so that both the writes and
          // the read-back are free of bank conflicts, then writes them out as
          // contiguous 512-byte rows (the 32 pixels are contiguous in NHWC).
          constexpr int CPX = COUT / 8;            // 16-byte chunks per pixel
          constexpr int ROWB = COUT * 2;           // bytes per pixel
          constexpr int PPL = 128 / ROWB;          // pixels per 128-byte bank window
          unsigned char* wb = s_out + warp * 32 * ROWB;
  #pragma unroll
          for (int c = 0; c < CPX; c++) {
            __align__(16) __half h[8];
  #pragma unroll
            for (int e = 0; e < 8; e++) {
              float v = __uint_as_float(accv[8 * c + e]);
              if (MODE == 0 || MODE == 4) {
                v += s_bias[8 * c + e];
                v = v > 0.f ? v : 0.f;
              } else if (MODE == 1) {
                const uint32_t word = (&mk[c].x)[e >> 1];
                const uint16_t bits = (uint16_t)((e & 1) ? (word >> 16) : (word & 0xFFFFu));
                // FP16 > 0: sign clear and not +0 (NaN cannot occur in a ReLU output)
                v = ((bits & 0x8000u) == 0 && bits != 0) ? v : 0.f;
              }
              h[e] = __float2half_rn(v);
            }
            if (MODE == 4) {
  #pragma unroll
              for (int e = 0; e < 8; e++) {
                const float fv = __half2float(h[e]);
                const float nb = __shfl_xor_sync(0xffffffffu, fv, 1);  // pixel x + 1 (even lanes)
                float acc = odd_row ? pacc[8 * c + e] + fv : fv;
                if (pair_x) acc = acc + nb;
                pacc[8 * c + e] = acc;
              }
              if (pool_row && (lane & 1) == 0 && x < W) {
                const float inv = 1.f / (float)((pair_x ? 2 : 1) * (odd_row ? 2 : 1));
                uint4 o;
                __half2* oh = reinterpret_cast<__half2*>(&o);
  #pragma unroll
                for (int k = 0; k < 4; k++)
                  oh[k] = __floats2half2_rn(pacc[8 * c + 2 * k] * inv, pacc[8 * c + 2 * k + 1] * inv);
                const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
                reinterpret_cast<uint4*>(pool + (((long long)p * Ho + y / 2) * (long long)Wo + x / 2) * COUT)[c] = o;
              }
            }
            const int phys = c ^ ((lane / PPL) & (CPX - 1));
            *reinterpret_cast<uint4*>(wb + lane * ROWB + phys * 16) = *reinterpret_cast<const uint4*>(h);
          }
          __syncwarp();
          const int xw = tx * TILE_M + warp * 32;  // the warp's first pixel
          __half* ow = out + (((long long)p * H + y) * (long long)W + xw) * COUT;
  #pragma unroll
          for (int k = 0; k < CPX; k++) {
            const int o = k * 512 + lane * 16;  // byte offset in the warp's 32 * ROWB bytes
            const int px = o / ROWB, ch = (o % ROWB) / 16;
            const int phys = ch ^ ((px / PPL) & (CPX - 1));
            const uint4 v = *reinterpret_cast<const uint4*>(wb + px * ROWB + phys * 16);
            if (xw + px < W) *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(ow) + o) = v;
          }
          __syncwarp();
        } else if (x < W) {
  #pragma unroll
          for (int j = 0; j < DN_MAX_SLOTS; j++) {
            const long long o = (((long long)p * DN_MAX_SLOTS + j) * H + y) * (long long)W + x;
            float v = __uint_as_float(accv[j]) + s_bias[j];
            vis[o] = 1.f / (1.f + __expf(-v));
            if (conf) {
              float c = __uint_as_float(accv[DN_MAX_SLOTS + j]) + s_bias[DN_MAX_SLOTS + j];
              conf[o] = 1.f / (1.f + __expf(-c));
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 5) {
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_ALLOC)
                 : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 4-D map over an NHWC activation [planes][H][W][cin] (FP16): box of 8
// channels x halo_px(dil) pixels x 1 row x 1 plane.
cudaError_t make_in_map(CUtensorMap* map, const __half* in, int planes, int H, int W, int cin, int dil) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)planes};
  cuuint64_t strides[3] = {(cuuint64_t)cin * 2, (cuuint64_t)W * cin * 2, (cuuint64_t)H * W * cin * 2};
  cuuint32_t box[4] = {8, (cuuint32_t)halo_px(dil), 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, const_cast<__half*>(in), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, int COUT, int MODE>
cudaError_t launch_conv(const __half* in, int planes, int H, int W, int dil, const void* w, const float* b, __half* out,
                        float* vis, float* conf, const __half* aux, __half* pool, int* err, cudaStream_t s,
                        int num_sms) {
  using SM = ConvSmem<CIN, COUT>;
  if (dil < 1 || dil > MAX_DIL) return cudaErrorInvalidValue;
  const int smem = SM::total(dil);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  static int attr_bytes[64] = {};  // per device ordinal: the largest size set so far
  static std::mutex attr_mu;       // batch lanes launch from several host threads
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> g(attr_mu);
    if (dev >= 64 || attr_bytes[dev] < smem) {
      e = cudaFuncSetAttribute(k_conv3x3_tc<CIN, COUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      if (dev < 64) attr_bytes[dev] = smem;
    }
  }
  CUtensorMap map;
  e = make_in_map(&map, in, planes, H, W, CIN, dil);
  if (e != cudaSuccess) return e;
  // Two waves of the CTAs that fit an SM (shared memory: 228 KB less 1 KB
  // reserved per CTA; TMEM: 512 columns); CTAs beyond the resident ones
  // start as others finish, which balances the segments better than one
  // resident wave (1.8x slower) or one CTA per segment (1.2x slower), and
  // a CTA loads its weights once for many segments.
  const int fit_smem = (228 * 1024) / (smem + 1024);
  const int fit_tmem = 512 / (NACC * acc_cols(COUT));
  const int resident = std::max(1, std::min(fit_smem, fit_tmem));
  const long long rows_per_col = (H + dil - 1) / dil;
  const long long nsegs = (long long)planes * ((W + TILE_M - 1) / TILE_M) * dil * ((rows_per_col + SEG - 1) / SEG);
  long long grid = std::min<long long>(nsegs, (long long)num_sms * 2 * resident);
  if (grid < 1) grid = 1;
  k_conv3x3_tc<CIN, COUT, MODE><<<(int)grid, CONV_THREADS, smem, s>>>(map, planes, H, W, dil, (const uint4*)w, b,
                                                                      out, vis, conf, aux, pool, err);
  return cudaGetLastError();
}

// 2x2 average pooling, [P][H][W][C] -> [P][ceil(H/2)][ceil(W/2)][C] FP16;
// an output pixel averages the input pixels of its 2x2 block that exist.
// One thread per 8 channels of one output pixel.
__global__ void k_pool2(const __half* __restrict__ in, __half* __restrict__ out, int P, int H, int W, int C) {
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2, CC = C / 8;
  const long long n = (long long)P * Ho * Wo * CC;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int cc = (int)(t % CC);
    long long q = t / CC;
    const int x = (int)(q % Wo);
    q /= Wo;
    const int y = (int)(q % Ho);
    const long long p = q / Ho;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int cnt = 0;
    for (int dy = 0; dy < 2; dy++)
      for (int dx = 0; dx < 2; dx++) {
        const int yy = 2 * y + dy, xx = 2 * x + dx;
        if (yy >= H || xx >= W) continue;
        const uint4 v = reinterpret_cast<const uint4*>(in + ((p * H + yy) * (long long)W + xx) * C)[cc];
        const __half2* h = reinterpret_cast<const __half2*>(&v);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          float2 f = __half22float2(h[k]);
          acc[2 * k] += f.x;
          acc[2 * k + 1] += f.y;
        }
        cnt++;
      }
    const float inv = 1.f / (float)cnt;
    uint4 o;
    __half2* oh = reinterpret_cast<__half2*>(&o);
#pragma unroll
    for (int k = 0; k < 4; k++) oh[k] = __floats2half2_rn(acc[2 * k] * inv, acc[2 * k + 1] * inv);
    reinterpret_cast<uint4*>(out + ((p * Ho + y) * (long long)Wo + x) * C)[cc] = o;
  }
}

// Nearest 2x upsampling of `low` ([P][ceil(H/2)][ceil(W/2)][C]) added to
// `skip` ([P][H][W][C]): out(y, x) = low(y / 2, x / 2) + skip(y, x), FP16.
__global__ void k_upadd(const __half* __restrict__ low, const __half* __restrict__ skip, __half* __restrict__ out,
                        int P, int H, int W, int C) {
  const int Hl = (H + 1) / 2, Wl = (W + 1) / 2, CC = C / 8;
  const long long n = (long long)P * H * W * CC;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int cc = (int)(t % CC);
    long long q = t / CC;
    const int x = (int)(q % W);
    q /= W;
    const int y = (int)(q % H);
    const long long p = q / H;
    const uint4 a = reinterpret_cast<const uint4*>(low + ((p * Hl + y / 2) * (long long)Wl + x / 2) * C)[cc];
    const uint4 b = reinterpret_cast<const uint4*>(skip)[t];
    uint4 o;
    const __half2* ah = reinterpret_cast<const __half2*>(&a);
    const __half2* bh = reinterpret_cast<const __half2*>(&b);
    __half2* oh = reinterpret_cast<__half2*>(&o);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float2 fa = __half22float2(ah[k]), fb = __half22float2(bh[k]);
      oh[k] = __floats2half2_rn(fa.x + fb.x, fa.y + fb.y);
    }
    reinterpret_cast<uint4*>(out)[t] = o;
  }
}

float half_to_float_host(uint16_t h) {
  __half_raw r;
  r.x = h;
  return __half2float(__half(r));
}

int level_dim(int n, int level) { return (n + (1 << level) - 1) >> level; }

}  // namespace

// Dispatch of the convolution shapes and epilogue modes the networks use
// (forward layers, and the transposed shapes of their backward data passes).
cudaError_t conv_launch(int cin, int cout, int mode, const __half* in, int planes, int H, int W, int dil,
                        const void* w, const float* b, __half* out, float* vis, float* conf, const __half* aux,
                        int* err, cudaStream_t s, int num_sms) {
#define RTB_CONV_CASE(CI, CO, M)                                                                         \
  if (cin == CI && cout == CO && mode == M)                                                              \
    return launch_conv<CI, CO, M>(in, planes, H, W, dil, w, b, out, vis, conf, aux, nullptr, err, s, num_sms);
#define RTB_CONV_SHAPE(CI, CO) RTB_CONV_CASE(CI, CO, 0) RTB_CONV_CASE(CI, CO, 1) RTB_CONV_CASE(CI, CO, 3)
  RTB_CONV_SHAPE(16, 16)
  RTB_CONV_SHAPE(16, 32)
  RTB_CONV_SHAPE(32, 16)
  RTB_CONV_SHAPE(32, 32)
  RTB_CONV_SHAPE(32, 64)
  RTB_CONV_SHAPE(64, 32)
  RTB_CONV_SHAPE(64, 64)
  RTB_CONV_CASE(16, 16, 2)
  RTB_CONV_CASE(32, 16, 2)
#undef RTB_CONV_SHAPE
#undef RTB_CONV_CASE
  return cudaErrorInvalidValue;
}

// A forward layer (bias + ReLU) whose output is also 2x2 average-pooled
// into `pool` ([planes][ceil(H/2)][ceil(W/2)][cout]), the bytes of
// pool2_launch on `out`.  Dilation 1 only; the shapes the network pools
// after (32 -> 32, 64 -> 64).
cudaError_t conv_pool_launch(int cin, int cout, const __half* in, int planes, int H, int W, const void* w,
                             const float* b, __half* out, __half* pool, int* err, cudaStream_t s, int num_sms) {
  if (cin == 32 && cout == 32)
    return launch_conv<32, 32, 4>(in, planes, H, W, 1, w, b, out, nullptr, nullptr, nullptr, pool, err, s, num_sms);
  if (cin == 64 && cout == 64)
    return launch_conv<64, 64, 4>(in, planes, H, W, 1, w, b, out, nullptr, nullptr, nullptr, pool, err, s, num_sms);
  return cudaErrorInvalidValue;
}

bool conv_pool_supported(int cin, int cout) { return cin == cout && (cin == 32 || cin == 64); }

bool conv_shape_supported(int cin, int cout) {
  static const int shapes[][2] = {{16, 16}, {16, 32}, {32, 16}, {32, 32}, {32, 64}, {64, 32}, {64, 64}};
  for (auto& sh : shapes)
    if (sh[0] == cin && sh[1] == cout) return true;
  return false;
}

cudaError_t pool2_launch(const __half* in, __half* out, int P, int H, int W, int C, cudaStream_t s, int num_sms) {
  const long long n = (long long)P * ((H + 1) / 2) * ((W + 1) / 2) * (C / 8);
  const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)num_sms * 16));
  k_pool2<<<blocks, 256, 0, s>>>(in, out, P, H, W, C);
  return cudaGetLastError();
}

cudaError_t upadd_launch(const __half* low, const __half* skip, __half* out, int P, int H, int W, int C,
                         cudaStream_t s, int num_sms) {
  const long long n = (long long)P * H * W * (C / 8);
  const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)num_sms * 16));
  k_upadd<<<blocks, 256, 0, s>>>(low, skip, out, P, H, W, C);
  return cudaGetLastError();
}

namespace {
// Reads version 1/2 blobs (a chain of convolutions) and version 3 blobs
// (an op list); fills ops (weights still on the host, in the blob's
// [cout][3][3][cin] FP16 layout, at w_off) or returns the reason.
struct ParsedOp {
  DnOp op;
  size_t w_off = 0;
};
std::string parse_blob(const unsigned char* p, size_t bytes, std::vector<ParsedOp>* out, int* rays, float* thr) {
  auto u32 = [&](size_t off) {
    uint32_t v;
    memcpy(&v, p + off, 4);
    return v;
  };
  if (!p || bytes < 12 || memcmp(p, "RTDN", 4) != 0) return "not a denoiser weight blob (magic RTDN)";
  const uint32_t ver = u32(4);
  if (ver < 1 || ver > 3) return "unsupported denoiser blob version";
  const uint32_t n = u32(8);
  if (n < 1 || n > 64) return "denoiser op count must be 1..64";
  size_t head = ver == 1 ? 12 : (ver == 2 ? 16 : 20);
  if (bytes < head) return "truncated denoiser blob";
  *rays = ver == 1 ? 1 : (int)u32(12);
  if (*rays < 1 || *rays > 16) return "denoiser rays per light must be 1..16";
  *thr = 1.0f;
  if (ver == 3) memcpy(thr, p + 16, 4);
  if (!(*thr >= 0.0f)) return "denoiser confidence threshold must be >= 0";
  const size_t rec = ver == 3 ? 28 : 16;
  size_t off = head + rec * n;
  if (bytes < off) return "truncated denoiser blob";
  std::vector<int> ch(1, FEAT_CHANNELS), lv(1, 0);  // per buffer
  out->assign(n, ParsedOp());
  for (uint32_t i = 0; i < n; i++) {
    DnOp& o = (*out)[i].op;
    const size_t r = head + rec * i;
    if (ver == 3) {
      o.kind = (int)u32(r);
      o.cin = (int)u32(r + 4);
      o.cout = (int)u32(r + 8);
      o.dil = (int)u32(r + 12);
      o.act = (int)u32(r + 16);
      o.src = (int)u32(r + 20);
      o.src2 = (int)u32(r + 24);
    } else {
      o.kind = DN_CONV;
      o.cin = (int)u32(r);
      o.cout = (int)u32(r + 4);
      o.dil = (int)u32(r + 8);
      o.act = (int)u32(r + 12);
      o.src = (int)i;
      o.src2 = -1;
    }
    const bool last = i + 1 == n;
    if (o.src < 0 || o.src > (int)i) return "denoiser op reads a buffer not yet written";
    if (o.kind == DN_CONV) {
      if (!conv_shape_supported(o.cin, o.cout)) return "unsupported denoiser convolution channel counts";
      if (o.cin != ch[o.src]) return "denoiser layer channel counts do not chain";
      if (o.dil < 1 || o.dil > MAX_DIL) return "denoiser dilation must be 1..64";
      if (o.act != (last ? 2 : 0)) return "denoiser layers must be ReLU, the last one sigmoid";
      o.level = lv[o.src];
    } else if (o.kind == DN_POOL) {
      if (o.cin != ch[o.src] || o.cout != o.cin) return "denoiser pooling must keep its channel count";
      if (lv[o.src] >= 4) return "denoiser pooling beyond level 4";
      o.level = lv[o.src] + 1;
    } else if (o.kind == DN_UPADD) {
      if (o.src2 < 0 || o.src2 > (int)i) return "denoiser op reads a buffer not yet written";
      if (lv[o.src] != lv[o.src2] + 1) return "denoiser upsampling must join adjacent levels";
      if (o.cin != ch[o.src] || o.cin != ch[o.src2] || o.cout != o.cin)
        return "denoiser upsampling must add equal channel counts";
      o.level = lv[o.src2];
    } else {
      return "unknown denoiser op kind";
    }
    if (last && (o.kind != DN_CONV || o.cout != 16 || o.level != 0))
      return "the last denoiser op must be a convolution writing 16 channels at full resolution";
    if (i == 0 && o.kind == DN_CONV && o.cin != FEAT_CHANNELS)
      return "the first denoiser layer must read 16 feature channels";
    ch.push_back(o.cout);
    lv.push_back(o.level);
  }
  for (uint32_t i = 0; i < n; i++) {
    ParsedOp& po = (*out)[i];
    if (po.op.kind != DN_CONV) continue;
    const size_t wbytes = (size_t)po.op.cout * 9 * po.op.cin * 2, bbytes = (size_t)po.op.cout * 4;
    if (bytes < off + wbytes + bbytes) return "truncated denoiser blob";
    po.w_off = off;
    off += wbytes + bbytes;
  }
  if (off != bytes) return "denoiser blob has trailing bytes";
  return std::string();
}
}  // namespace

std::string denoise_load(const void* blob, size_t bytes, DenoiseNet* net) {
  denoise_free(net);
  const unsigned char* p = static_cast<const unsigned char*>(blob);
  std::vector<ParsedOp> ops;
  int rays = 1;
  float thr = 1.0f;
  std::string perr = parse_blob(p, bytes, &ops, &rays, &thr);
  if (!perr.empty()) return perr;
  std::vector<void*> allocs;
  auto fail = [&](const std::string& m) {
    for (void* a : allocs) cudaFree(a);
    return m;
  };
  size_t params = 0;
  std::vector<DnOp> L;
  for (ParsedOp& po : ops) {
    DnOp o = po.op;
    if (o.kind == DN_CONV) {
      const int cin = o.cin, cout = o.cout, K = 9 * cin;
      const size_t wbytes = (size_t)cout * K * 2, bbytes = (size_t)cout * 4;
      const uint16_t* w = reinterpret_cast<const uint16_t*>(p + po.w_off);
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
          cudaMemcpy(db, p + po.w_off + wbytes, bbytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail("uploading denoiser weights failed");
      o.w = dw;
      o.b = db;
      params += (size_t)cout * K + cout;
    }
    L.push_back(o);
  }
  net->ops = L;
  net->allocs = allocs;
  net->param_count = params;
  net->rays_per_light = rays;
  net->conf_threshold = thr;
  // version 3 networks output an error estimate per slot (channels 2, 3)
  net->has_conf = memcmp(p + 4, "\x03\x00\x00\x00", 4) == 0;
  return std::string();
}

void denoise_free(DenoiseNet* net) {
  for (void* a : net->allocs) cudaFree(a);
  net->allocs.clear();
  net->ops.clear();
  net->param_count = 0;
  net->rays_per_light = 1;
  net->has_conf = false;
  net->conf_threshold = 1.0f;
}

size_t denoise_scratch_halves(const DenoiseNet& net, int planes, int H, int W) {
  size_t n = 0;
  for (size_t i = 0; i + 1 < net.ops.size(); i++) {
    const DnOp& o = net.ops[i];
    n += (size_t)planes * level_dim(H, o.level) * level_dim(W, o.level) * o.cout;
    n = (n + 127) & ~(size_t)127;  // 256-byte aligned buffers
  }
  return std::max<size_t>(n, 128);
}

int denoise_run(const DenoiseNet& net, const __half* feat, int planes, int H, int W, __half* arena, float* vis,
                float* conf, int* err, cudaStream_t s, int num_sms, cudaError_t* launch_err) {
  std::vector<const __half*> buf(net.ops.size() + 1, nullptr);
  buf[0] = feat;
  size_t off = 0;
  int launches = 0;
  *launch_err = cudaSuccess;
  for (size_t i = 0; i < net.ops.size(); i++) {
    const DnOp& o = net.ops[i];
    const int h = level_dim(H, o.level), w = level_dim(W, o.level);
    __half* out = nullptr;
    if (i + 1 < net.ops.size()) {
      out = arena + off;
      off += (size_t)planes * h * w * o.cout;
      off = (off + 127) & ~(size_t)127;
    }
    cudaError_t e;
    // a forward layer whose output the next op pools: one launch writes both
    const DnOp* np = i + 1 < net.ops.size() ? &net.ops[i + 1] : nullptr;
    if (o.kind == DN_CONV && o.act == 0 && o.dil == 1 && np && np->kind == DN_POOL && np->src == (int)i + 1 &&
        i + 2 < net.ops.size() && conv_pool_supported(o.cin, o.cout)) {
      __half* pooled = arena + off;
      off += (size_t)planes * level_dim(H, np->level) * level_dim(W, np->level) * np->cout;
      off = (off + 127) & ~(size_t)127;
      e = conv_pool_launch(o.cin, o.cout, buf[o.src], planes, h, w, o.w, o.b, out, pooled, err, s, num_sms);
      launches++;
      if (e != cudaSuccess) {
        *launch_err = e;
        return launches;
      }
      buf[i + 1] = out;
      buf[i + 2] = pooled;
      i++;
      continue;
    }
    if (o.kind == DN_CONV) {
      if (o.act == 2)
        e = conv_launch(o.cin, o.cout, 2, buf[o.src], planes, h, w, o.dil, o.w, o.b, nullptr, vis,
                        net.has_conf ? conf : nullptr, nullptr, err, s, num_sms);
      else
        e = conv_launch(o.cin, o.cout, 0, buf[o.src], planes, h, w, o.dil, o.w, o.b, out, nullptr, nullptr, nullptr,
                        err, s, num_sms);
    } else if (o.kind == DN_POOL) {
      e = pool2_launch(buf[o.src], out, planes, level_dim(H, o.level - 1), level_dim(W, o.level - 1), o.cin, s,
                       num_sms);
    } else {
      e = upadd_launch(buf[o.src], buf[o.src2], out, planes, h, w, o.cin, s, num_sms);
    }
    launches++;
    if (e != cudaSuccess) {
      *launch_err = e;
      return launches;
    }
    buf[i + 1] = out;
  }
  return launches;
}

}  // namespace rtb
