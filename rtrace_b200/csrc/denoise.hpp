// Learned soft-shadow denoiser: a stack of dilated 3x3 convolutions over the
// primary hits' feature image, run as tcgen05 implicit GEMMs (FP16 operands,
// FP32 accumulation in tensor memory).  This is an extension: the reference
// always casts 16 shadow rays per disk light and has no denoiser.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <vector>

namespace rtb {

// Channels of the feature image (one 16-channel FP16 pixel per primary
// sample).  The first two disk lights of a scene are the denoised "slots".
enum {
  FEAT_VALID = 0,   // 1 where the primary ray hit
  FEAT_DEPTH = 1,   // camera distance d mapped to d / (d + 4)
  FEAT_NX = 2,      // world normal
  FEAT_SLOT0 = 5,   // per slot j, base FEAT_SLOT0 + 4 j:
  FEAT_SLOT_STRIDE = 4,  //   +0 visibility of the cast samples (visible / samples)
                         //   +1 max(n . l, 0) towards the light centre
                         //   +2 light radius / centre distance, clamped to [0, 1]
                         //   +3 1 (slot present)
  FEAT_PIXEL_VIS = 13,   // per slot j, FEAT_PIXEL_VIS + j: the mean cast-ray visibility over
                         // the pixel's samples that hit (every sample plane of the pixel)
  FEAT_CHANNELS = 16,
  DN_MAX_SLOTS = 2,
};

// Error bit set when a wait on the tensor cores ran out (the renderer's
// error word; its other bits are the ERR_* of dscene.cuh).
constexpr int DN_ERR_WAIT = 16;

// One operation of the network.  Buffer 0 is the feature image; op i
// writes buffer i + 1.  Resolution level l has ceil(H / 2^l) x ceil(W / 2^l)
// pixels per plane; every buffer is FP16 NHWC.
enum { DN_CONV = 0, DN_POOL = 1, DN_UPADD = 2 };
struct DnOp {
  int kind = DN_CONV;
  int cin = 0, cout = 0, dil = 1, act = 0;  // conv act: 0 ReLU, 2 sigmoid outputs (last op only)
  int src = 0, src2 = -1;                   // input buffer(s); upadd: src is the coarse one, src2 the skip
  int level = 0;                            // level of the output
  void* w = nullptr;                        // conv: weights in the tensor-core operand layout
  float* b = nullptr;
};

struct DenoiseNet {
  std::vector<DnOp> ops;
  std::vector<void*> allocs;
  size_t param_count = 0;
  int rays_per_light = 1;  // disk-light rays per primary hit the network was trained on
  bool has_conf = false;   // the output holds an error estimate per slot (channels 2, 3)
  float conf_threshold = 1.0f;  // default fallback threshold stored with the weights
  bool loaded() const { return !ops.empty(); }
};

// Parses and uploads a weight blob (format in include/rtrace_gpu.h next to
// rt_denoiser_load).  Returns an empty string on success, else the reason.
std::string denoise_load(const void* blob, size_t bytes, DenoiseNet* net);
void denoise_free(DenoiseNet* net);

// Halves of activation scratch denoise_run needs for planes x H x W.
size_t denoise_scratch_halves(const DenoiseNet& net, int planes, int H, int W);

// Runs the network on feat ([planes][H][W][16] FP16) and writes the
// visibility estimate of each slot to vis ([planes][2][H][W] float) and,
// when the network has them and conf is not null, its error estimates to
// conf (same layout).  arena holds denoise_scratch_halves() halves.  err
// receives a nonzero code if a wait on the tensor cores ran out.  Returns
// the number of launches.
int denoise_run(const DenoiseNet& net, const __half* feat, int planes, int H, int W, __half* arena, float* vis,
                float* conf, int* err, cudaStream_t s, int num_sms, cudaError_t* launch_err);

// The building blocks, also used by training (rtrace_b200/csrc/dn_train.cu).
// conv_launch: one 3x3 convolution (see k_conv3x3_tc for the epilogue
// modes) of an FP16 NHWC tensor [planes][H][W][cin]; w in the tensor-core
// operand layout.  cudaErrorInvalidValue for an unsupported shape or mode.
cudaError_t conv_launch(int cin, int cout, int mode, const __half* in, int planes, int H, int W, int dil,
                        const void* w, const float* b, __half* out, float* vis, float* conf, const __half* aux,
                        int* err, cudaStream_t s, int num_sms);
bool conv_shape_supported(int cin, int cout);
cudaError_t pool2_launch(const __half* in, __half* out, int P, int H, int W, int C, cudaStream_t s, int num_sms);
cudaError_t upadd_launch(const __half* low, const __half* skip, __half* out, int P, int H, int W, int C,
                         cudaStream_t s, int num_sms);

}  // namespace rtb
