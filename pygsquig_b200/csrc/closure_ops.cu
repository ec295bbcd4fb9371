// closure_ops.cu -- the small kernels of the learned closure around the
// tensor-core convolutions: the 1-channel first and last layers (3x3, 1 -> 64
// and 64 -> 1, CUDA cores), their gradients, bias gradients, the MSE loss,
// Adam, and the weight re-layouts the tensor-core kernels read.
//
// Layouts: NHWC; "halo'd" tensors are [B][H+2][W+2][C] with a one-pixel
// circular halo.  Reductions over pixels write per-block partial sums that a
// second kernel adds in a fixed order (bitwise reproducible).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sqg_closure.h"

namespace {

thread_local std::string g_err;
int ofail(const std::string& m) {
  g_err = m;
  return 1;
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
__device__ __forceinline__ size_t padidx(int b, int y, int x, int H, int W) {
  return ((size_t)b * (H + 2) + (y + 1)) * (W + 2) + (x + 1);
}

// Writes the 64 BF16 channels of interior pixel (b, y, x) and its halo copies.
__device__ __forceinline__ void put_halo(__nv_bfloat16* out, int H, int W, int b, int y, int x, const float* v) {
  int ys[2] = {y + 1, -1}, xs[2] = {x + 1, -1};
  if (y == 0) ys[1] = H + 1;
  if (y == H - 1) ys[1] = 0;
  if (x == 0) xs[1] = W + 1;
  if (x == W - 1) xs[1] = 0;
  uint4 pk[8];
#pragma unroll
  for (int i = 0; i < 32; ++i) reinterpret_cast<__nv_bfloat162*>(pk)[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  for (int a = 0; a < 2; ++a) {
    if (ys[a] < 0) continue;
    for (int c = 0; c < 2; ++c) {
      if (xs[c] < 0) continue;
      uint4* d = reinterpret_cast<uint4*>(out + (((size_t)b * (H + 2) + ys[a]) * (W + 2) + xs[c]) * 64);
#pragma unroll
      for (int i = 0; i < 8; ++i) d[i] = pk[i];
    }
  }
}

// Layer 1 forward: z = conv3x3(x; w[9][64]) + b (1 -> 64), a = gelu(z).
__global__ void k_conv_in(int B, int H, int W, const float* __restrict__ x, const float* __restrict__ w,
                          const float* __restrict__ bias, __nv_bfloat16* __restrict__ z,
                          __nv_bfloat16* __restrict__ a_pad) {
  const size_t n = (size_t)B * H * W;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int xx = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((size_t)W * H));
    float xv[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int yy = wrap(y + t / 3 - 1, H), xw = wrap(xx + t % 3 - 1, W);
      xv[t] = x[((size_t)b * H + yy) * W + xw];
    }
    float zf[64], af[64];
#pragma unroll 8
    for (int c = 0; c < 64; ++c) {
      float s = bias[c];
#pragma unroll
      for (int t = 0; t < 9; ++t) s += xv[t] * w[t * 64 + c];
      const float zb = __bfloat162float(__float2bfloat16_rn(s));
      zf[c] = zb;
      af[c] = gelu(zb);
    }
    uint4* zo = reinterpret_cast<uint4*>(z + p * 64);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      uint4 v;
      __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
      for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(zf[8 * i + 2 * j], zf[8 * i + 2 * j + 1]);
      zo[i] = v;
    }
    put_halo(a_pad, H, W, b, y, xx, af);
  }
}

// Last layer forward: y = conv3x3(a; w[9][64]) + b (64 -> 1), FP32 output.
__global__ void k_conv_out(int B, int H, int W, const __nv_bfloat16* __restrict__ a_pad, const float* __restrict__ w,
                           const float* __restrict__ bias, float* __restrict__ y) {
  __shared__ float sw[9 * 64];
  for (int i = threadIdx.x; i < 9 * 64; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  const size_t n = (size_t)B * H * W;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int xx = (int)(p % W), yy = (int)((p / W) % H), b = (int)(p / ((size_t)W * H));
    float s = bias[0];
    for (int t = 0; t < 9; ++t) {
      const uint4* src = reinterpret_cast<const uint4*>(a_pad + padidx(b, yy + t / 3 - 1, xx + t % 3 - 1, H, W) * 64);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const uint4 v = src[i];
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float2 f = __bfloat1622float2(h[j]);
          s += f.x * sw[t * 64 + 8 * i + 2 * j] + f.y * sw[t * 64 + 8 * i + 2 * j + 1];
        }
      }
    }
    y[p] = s;
  }
}

// Last layer backward, data part: g_a[q][c] = sum_t gy[q - off_t] w[t][c],
// then times gelu'(z[q][c]) -> halo'd BF16 gradient of the layer-5 pre-activation.
__global__ void k_conv_out_dgrad(int B, int H, int W, const float* __restrict__ gy, const float* __restrict__ w,
                                 const __nv_bfloat16* __restrict__ z, __nv_bfloat16* __restrict__ gz_pad) {
  __shared__ float sw[9 * 64];
  for (int i = threadIdx.x; i < 9 * 64; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  const size_t n = (size_t)B * H * W;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int xx = (int)(q % W), yy = (int)((q / W) % H), b = (int)(q / ((size_t)W * H));
    float g9[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int py = wrap(yy - (t / 3 - 1), H), px = wrap(xx - (t % 3 - 1), W);
      g9[t] = gy[((size_t)b * H + py) * W + px];
    }
    const uint4* zs = reinterpret_cast<const uint4*>(z + q * 64);
    float out[64];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint4 v = zs[i];
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 zz = __bfloat1622float2(h[j]);
        const int c = 8 * i + 2 * j;
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          s0 += g9[t] * sw[t * 64 + c];
          s1 += g9[t] * sw[t * 64 + c + 1];
        }
        out[c] = s0 * gelu_grad(zz.x);
        out[c + 1] = s1 * gelu_grad(zz.y);
      }
    }
    put_halo(gz_pad, H, W, b, yy, xx, out);
  }
}

// Per-block partial sums of the small-layer gradients (fixed grid).
//  mode 0 (last layer):  part[blk][t*64 + c] = sum_p gy[p] a[p + t][c]; part[blk][576] = sum gy
//  mode 1 (first layer): part[blk][t*64 + c] = sum_p gz[p][c] x[p + t];  part[blk][576 + c] = sum gz[.][c]
//  mode 2 (bias of a middle layer): part[blk][c] = sum_p gz[p][c]
constexpr int kRedBlocks = 296;
constexpr int kRedStride = 9 * 64 + 64;
__global__ void k_small_grad_partial(int mode, int B, int H, int W, const float* __restrict__ gy,
                                     const __nv_bfloat16* __restrict__ a_pad, const float* __restrict__ x,
                                     const __nv_bfloat16* __restrict__ gz_pad, float* __restrict__ part) {
  __shared__ float acc[kRedStride];
  for (int i = threadIdx.x; i < kRedStride; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  const size_t n = (size_t)B * H * W;
  // each thread keeps its own channel slice: thread (c = threadIdx.x % 64) accumulates channel c
  const int c = threadIdx.x & 63, lanes = blockDim.x / 64, sub = threadIdx.x / 64;
  float loc[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) loc[i] = 0.f;
  for (size_t p = blockIdx.x * (size_t)lanes + sub; p < n; p += (size_t)gridDim.x * lanes) {
    const int xx = (int)(p % W), yy = (int)((p / W) % H), b = (int)(p / ((size_t)W * H));
    if (mode == 0) {
      const float g = gy[p];
#pragma unroll
      for (int t = 0; t < 9; ++t)
        loc[t] += g * __bfloat162float(a_pad[padidx(b, yy + t / 3 - 1, xx + t % 3 - 1, H, W) * 64 + c]);
      if (c == 0) loc[9] += g;
    } else if (mode == 1) {
      const float g = __bfloat162float(gz_pad[padidx(b, yy, xx, H, W) * 64 + c]);
#pragma unroll
      for (int t = 0; t < 9; ++t) loc[t] += g * x[((size_t)b * H + wrap(yy + t / 3 - 1, H)) * W + wrap(xx + t % 3 - 1, W)];
      loc[9] += g;
    } else {
      loc[9] += __bfloat162float(gz_pad[padidx(b, yy, xx, H, W) * 64 + c]);
    }
  }
  // fixed-order combination of the block's threads
  for (int s = 0; s < lanes; ++s) {
    if (sub == s) {
      for (int t = 0; t < 9; ++t) acc[t * 64 + c] += loc[t];
      acc[576 + c] += loc[9];
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < kRedStride; i += blockDim.x) part[(size_t)blockIdx.x * kRedStride + i] = acc[i];
}

__global__ void k_small_grad_final(int nblk, const float* __restrict__ part, float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kRedStride; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * kRedStride + i];
    out[i] = s;
  }
}

// MSE loss and its gradient: gy = 2 (y - t) / n; part[blk] = sum (y - t)^2.
__global__ void k_mse(size_t n, const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ gy,
                      float* __restrict__ part) {
  __shared__ float red[256];
  float s = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    gy[i] = 2.f * d / (float)n;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (bias-corrected) on a flat FP32 parameter vector.
__global__ void k_adam(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 weights of a middle layer for the tensor cores: forward [t][co][ci]
// as stored, and the backward-data form wb[8 - t][ci][co] (flipped taps,
// swapped channels).
__global__ void k_weights_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                               __nv_bfloat16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 9 * 64 * 64) return;
  const int t = i / 4096, co = (i / 64) % 64, ci = i % 64;
  const __nv_bfloat16 h = __float2bfloat16_rn(w[i]);
  wf[i] = h;
  wb[((size_t)(8 - t) * 64 + ci) * 64 + co] = h;
}

// FP32 [B][H][W] -> halo'd scalar copy is not needed: layers read x with wrap.

}  // namespace

extern "C" {

int closure_conv_in(int32_t B, int32_t H, int32_t W, const float* x, const float* w, const float* bias, void* z,
                    void* a_pad, void* stream) {
  if (!x || !w || !bias || !z || !a_pad) return ofail("closure_conv_in: null pointer");
  k_conv_in<<<592, 128, 0, (cudaStream_t)stream>>>(B, H, W, x, w, bias, (__nv_bfloat16*)z, (__nv_bfloat16*)a_pad);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_conv_in: launch failed");
}

int closure_conv_out(int32_t B, int32_t H, int32_t W, const void* a_pad, const float* w, const float* bias, float* y,
                     void* stream) {
  if (!a_pad || !w || !bias || !y) return ofail("closure_conv_out: null pointer");
  k_conv_out<<<592, 128, 0, (cudaStream_t)stream>>>(B, H, W, (const __nv_bfloat16*)a_pad, w, bias, y);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_conv_out: launch failed");
}

int closure_conv_out_dgrad(int32_t B, int32_t H, int32_t W, const float* gy, const float* w, const void* z,
                           void* gz_pad, void* stream) {
  if (!gy || !w || !z || !gz_pad) return ofail("closure_conv_out_dgrad: null pointer");
  k_conv_out_dgrad<<<592, 128, 0, (cudaStream_t)stream>>>(B, H, W, gy, w, (const __nv_bfloat16*)z,
                                                          (__nv_bfloat16*)gz_pad);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_conv_out_dgrad: launch failed");
}

int closure_small_grad(int32_t mode, int32_t B, int32_t H, int32_t W, const float* gy, const void* a_pad,
                       const float* x, const void* gz_pad, float* partials, float* out, void* stream) {
  if (!partials || !out) return ofail("closure_small_grad: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  k_small_grad_partial<<<kRedBlocks, 256, 0, st>>>(mode, B, H, W, gy, (const __nv_bfloat16*)a_pad, x,
                                                   (const __nv_bfloat16*)gz_pad, partials);
  k_small_grad_final<<<3, 256, 0, st>>>(kRedBlocks, partials, out);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_small_grad: launch failed");
}

int closure_mse(int64_t n, const float* y, const float* t, float* gy, float* partials, void* stream) {
  if (!y || !t || !gy || !partials) return ofail("closure_mse: null pointer");
  k_mse<<<296, 256, 0, (cudaStream_t)stream>>>((size_t)n, y, t, gy, partials);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_mse: launch failed");
}

int closure_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                 int32_t step, void* stream) {
  if (!p || !g || !m || !v || step < 1) return ofail("closure_adam: bad arguments");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<296, 256, 0, (cudaStream_t)stream>>>((size_t)n, p, g, m, v, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_adam: launch failed");
}

int closure_weights_bf16(const float* w, void* wf, void* wb, void* stream) {
  if (!w || !wf || !wb) return ofail("closure_weights_bf16: null pointer");
  k_weights_bf16<<<(9 * 4096 + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16*)wf, (__nv_bfloat16*)wb);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_weights_bf16: launch failed");
}

const char* closure_ops_last_error_string(void) { return g_err.c_str(); }

}  // extern "C"
