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

/* Weight gradient of closure_conv64 on tcgen05 tensor cores:
 * dw[t][co][ci] = sum_p act[p + off_t][ci] * grad[p][co] over all interior
 * pixels p.  act_pad, grad_pad: BF16 [B][H+2][W+2][64] halo'd (only the
 * interior of grad_pad is read).  partials: FP32 scratch of nparts * 5 * 128
 * * 64 floats (nparts persistent CTAs each sum a range of pixel blocks; the
 * partial sums are added in a fixed order).  dw: FP32 [9][64][64]. */
int closure_wgrad64(int32_t B, int32_t H, int32_t W, const void* act_pad, const void* grad_pad, float* partials,
                    int32_t nparts, float* dw, uint32_t* err, void* stream);

/* CUDA-core kernels of the 1-channel layers and the training step
 * (W a multiple of 32, H >= 2; a warp owns 32 pixels of a row, a lane a
 * channel pair).
 * conv_in:  z = conv3x3(in_scale x; w[9][64]) + bias (1 -> 64); z BF16
 *           [B][H][W][64], a_pad = gelu(z) BF16 halo'd.  x: FP32 [B][H][W].
 * conv_out: y = out_scale (conv3x3(a; w[9][64]) + bias[0]) (64 -> 1), y FP32
 *           [B][H][W].  (The scales fold an input / output normalisation
 *           into the layers; training passes 1.)
 * conv_out_dgrad: gz_pad = (sum_t gy[q - off_t] w[t][c]) * gelu'(z[q][c]).
 * small_grad: mode 0 -> out[t*64+c] = sum_p gy[p] a[p+off_t][c], out[576] = sum gy;
 *             mode 1 -> out[t*64+c] = sum_p gz[p][c] x[p+off_t], out[576+c] = sum_p gz[p][c];
 *             mode 2 -> out[576+c] = sum_p gz[p][c].  partials: 296 * 640 floats.
 * mse: gy = 2 (y - t) / n; partials[296] = per-block sums of (y - t)^2.
 * adam: bias-corrected Adam step number `step` (>= 1) on a flat FP32 vector.
 * weights_bf16: wf[t][co][ci] = w, wb[8-t][ci][co] = w (backward-data form). */
int closure_conv_in(int32_t B, int32_t H, int32_t W, float in_scale, const float* x, const float* w, const float* bias,
                    void* z, void* a_pad, void* stream);
int closure_conv_out(int32_t B, int32_t H, int32_t W, float out_scale, const void* a_pad, const float* w,
                     const float* bias, float* y, void* stream);
int closure_conv_out_dgrad(int32_t B, int32_t H, int32_t W, const float* gy, const float* w, const void* z,
                           void* gz_pad, void* stream);
int closure_small_grad(int32_t mode, int32_t B, int32_t H, int32_t W, const float* gy, const void* a_pad,
                       const float* x, const void* gz_pad, float* partials, float* out, void* stream);
int closure_mse(int64_t n, const float* y, const float* t, float* gy, float* partials, void* stream);
int closure_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                 int32_t step, void* stream);
int closure_weights_bf16(const float* w, void* wf, void* wb, void* stream);
const char* closure_ops_last_error_string(void);

const char* closure_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif /* SQG_CLOSURE_H */
