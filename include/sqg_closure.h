/*
 * sqg_closure.h -- C ABI of the learned subgrid closure kernels in libsqg.
 *
 * No counterpart in the reference (the reference has no learned closure);
 * these kernels implement the 6-layer 3x3 CNN closure, with BF16 tensor-core
 * (tcgen05) convolutions accumulating in FP32.
 *
 * Tensors are NHWC.  "Halo'd" tensors are [B][H+2][W+2][C] with a one-pixel
 * circular halo (periodic domain); the kernels that write them also write the
 * halo copies.
 */
#ifndef SQG_CLOSURE_H
#define SQG_CLOSURE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CLOSURE_EPI_FWD = 0,   /* z = conv + bias -> out_z (BF16); gelu(z) -> out_pad (BF16, halo'd) */
  CLOSURE_EPI_DGRAD = 1, /* g = conv * gelu'(zprev) -> out_pad (BF16, halo'd)                  */
  CLOSURE_EPI_LIN = 2    /* conv + bias -> out_f32 (FP32, [B][H][W][64])                       */
};

/* 3x3 convolution, 64 -> 64 channels, circular padding, on tcgen05 tensor
 * cores.  act_pad: BF16 [B][H+2][W+2][64] halo'd input.  weights: BF16
 * [9][64 out][64 in] (tap t = 3 (dy+1) + (dx+1)).  W must be a multiple of
 * 128.  err: device uint32 flag set non-zero if a bounded wait timed out.
 * grid <= 0 picks one persistent CTA per SM.  Asynchronous on stream. */
int closure_conv64(int32_t B, int32_t H, int32_t W, int32_t mode, const void* act_pad, const void* weights,
                   const float* bias, const void* zprev, void* out_pad, void* out_z, float* out_f32,
                   uint32_t* err, int32_t grid, void* stream);

const char* closure_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif /* SQG_CLOSURE_H */
