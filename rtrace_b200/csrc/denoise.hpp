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
  FEAT_CHANNELS = 16,
  DN_MAX_SLOTS = 2,
};

// Error bit set when a wait on the tensor cores ran out (the renderer's
// error word; its other bits are the ERR_* of dscene.cuh).
constexpr int DN_ERR_WAIT = 16;

struct DnLayer {
  int cin = 0, cout = 0, dil = 1, act = 0;  // act: 0 ReLU, 2 sigmoid (last layer)
  void* w = nullptr;                        // weights in the tensor-core operand layout
  float* b = nullptr;
};

struct DenoiseNet {
  std::vector<DnLayer> layers;
  std::vector<void*> allocs;
  size_t param_count = 0;
  int rays_per_light = 1;  // disk-light rays per primary hit the network was trained on
  bool loaded() const { return !layers.empty(); }
};

// Parses and uploads a weight blob (format in include/rtrace_gpu.h next to
// rt_denoiser_load).  Returns an empty string on success, else the reason.
std::string denoise_load(const void* blob, size_t bytes, DenoiseNet* net);
void denoise_free(DenoiseNet* net);

// Runs the network on feat ([planes][H][W][16] FP16) and writes the
// visibility estimate of each slot to vis ([planes][2][H][W] float).
// act0/act1 hold planes*H*W*32 halves each.  err receives a nonzero code if
// a wait on the tensor cores ran out.  Returns the number of launches.
int denoise_run(const DenoiseNet& net, const __half* feat, int planes, int H, int W, __half* act0, __half* act1,
                float* vis, int* err, cudaStream_t s, int num_sms, cudaError_t* launch_err);

}  // namespace rtb
