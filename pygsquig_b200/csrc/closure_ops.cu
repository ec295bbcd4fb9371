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
#include "closure_act.cuh"
#include "pdl.cuh"

namespace {

thread_local std::string g_err;
int ofail(const std::string& m) {
  g_err = m;
  return 1;
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
__device__ __forceinline__ size_t padidx(int b, int y, int x, int H, int W) {
  return ((size_t)b * (H + 2) + (y + 1)) * (W + 2) + (x + 1);
}

// Work item of one warp: 32 consecutive pixels of one image row (W is a
// multiple of 32); lane l owns the channel pair (2l, 2l + 1), so every
// per-pixel access of a 64-channel tensor is one coalesced 128-byte row.
constexpr int kChunk = 32;
constexpr int kWarps = 8;  // warps per block of the chunked kernels

struct Chunk {
  int b, y, x0;
  size_t p0;  // linear index of the first pixel
};
__device__ __forceinline__ Chunk chunk_of(size_t ch, int H, int W) {
  Chunk c;
  c.p0 = ch * kChunk;
  c.x0 = (int)(c.p0 % W);
  const size_t r = c.p0 / W;
  c.y = (int)(r % H);
  c.b = (int)(r / H);
  return c;
}

// Rows y-1, y, y+1 (circular) of a scalar field, columns x0-1 .. x0+32, into s[3][34].
__device__ __forceinline__ void stage_rows(float (*s)[34], const float* __restrict__ f, int H, int W, const Chunk& c,
                                           int lane) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float* row = f + ((size_t)c.b * H + wrap(c.y + r - 1, H)) * W;
    s[r][lane + 1] = row[c.x0 + lane];
    if (lane == 0) s[r][0] = row[wrap(c.x0 - 1, W)];
    if (lane == 1) s[r][33] = row[wrap(c.x0 + kChunk, W)];
  }
  __syncwarp();
}

// The lane's channel pair of interior pixel (b, y, x) and its circular halo copies.
__device__ __forceinline__ void put2(__nv_bfloat16* out, int H, int W, int b, int y, int x, int lane,
                                     __nv_bfloat162 v) {
  const int Hp = H + 2, Wp = W + 2;
  const int y2 = (y == 0) ? H + 1 : (y == H - 1 ? 0 : -1);
  const int x2 = (x == 0) ? W + 1 : (x == W - 1 ? 0 : -1);
  reinterpret_cast<__nv_bfloat162*>(out + (((size_t)b * Hp + y + 1) * Wp + x + 1) * 64)[lane] = v;
  if (y2 >= 0) reinterpret_cast<__nv_bfloat162*>(out + (((size_t)b * Hp + y2) * Wp + x + 1) * 64)[lane] = v;
  if (x2 >= 0) {
    reinterpret_cast<__nv_bfloat162*>(out + (((size_t)b * Hp + y + 1) * Wp + x2) * 64)[lane] = v;
    if (y2 >= 0) reinterpret_cast<__nv_bfloat162*>(out + (((size_t)b * Hp + y2) * Wp + x2) * 64)[lane] = v;
  }
}

__device__ __forceinline__ float2 ld2(const __nv_bfloat16* t, size_t pix, int lane) {
  return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(t + pix * 64)[lane]);
}

// After the call lane l holds, in v[0], the sum over all lanes of their v[l].
__device__ __forceinline__ float reduce_scatter32(float (&v)[32], int lane) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < off; ++i) {
      const float send = upper ? v[i] : v[i + off];
      const float keep = upper ? v[i + off] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  return v[0];
}

// The 8-channel variant of put2: lane group g owns channels 8g .. 8g+7.
__device__ __forceinline__ void put8(__nv_bfloat16* out, int H, int W, int b, int y, int x, int g, uint4 v) {
  const int Hp = H + 2, Wp = W + 2;
  const int y2 = (y == 0) ? H + 1 : (y == H - 1 ? 0 : -1);
  const int x2 = (x == 0) ? W + 1 : (x == W - 1 ? 0 : -1);
  reinterpret_cast<uint4*>(out + (((size_t)b * Hp + y + 1) * Wp + x + 1) * 64)[g] = v;
  if (y2 >= 0) reinterpret_cast<uint4*>(out + (((size_t)b * Hp + y2) * Wp + x + 1) * 64)[g] = v;
  if (x2 >= 0) {
    reinterpret_cast<uint4*>(out + (((size_t)b * Hp + y + 1) * Wp + x2) * 64)[g] = v;
    if (y2 >= 0) reinterpret_cast<uint4*>(out + (((size_t)b * Hp + y2) * Wp + x2) * 64)[g] = v;
  }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 v;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return v;
}

// Layer 1 forward: z = conv3x3(in_scale x; w[9][64]) + b (1 -> 64), a = gelu(z).
// A warp takes its 32-pixel chunk four pixels at a time: lane l computes
// pixel l / 8 of the four, channels 8 (l % 8) .. +7, and writes them as one
// 16-byte store per tensor (a warp store covers 512 contiguous bytes).
__global__ void __launch_bounds__(kWarps * 32) k_conv_in(int B, int H, int W, float in_scale, const float* __restrict__ x,
                                                         const float* __restrict__ w, const float* __restrict__ bias,
                                                         __nv_bfloat16* __restrict__ z, __nv_bfloat16* __restrict__ a_pad) {
  __shared__ float stg[kWarps][3][34];
  pdl_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane >> 3, g = lane & 7;
  float wr[9][8], b8[8];
#pragma unroll
  for (int t = 0; t < 9; ++t)
#pragma unroll
    for (int i = 0; i < 8; ++i) wr[t][i] = w[t * 64 + 8 * g + i] * in_scale;
#pragma unroll
  for (int i = 0; i < 8; ++i) b8[i] = bias[8 * g + i];
  const size_t n_chunks = (size_t)B * H * W / kChunk;
  for (size_t ch = (size_t)blockIdx.x * kWarps + warp; ch < n_chunks; ch += (size_t)gridDim.x * kWarps) {
    const Chunk c = chunk_of(ch, H, W);
    __syncwarp();
    stage_rows(stg[warp], x, H, W, c, lane);
#pragma unroll 2
    for (int q = 0; q < kChunk / 4; ++q) {
      const int j = 4 * q + sub;
      float sv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) sv[i] = b8[i];
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const float xv = stg[warp][t / 3][j + t % 3];
#pragma unroll
        for (int i = 0; i < 8; ++i) sv[i] += xv * wr[t][i];
      }
      const uint4 zb = pack8(sv);
      reinterpret_cast<uint4*>(z + (c.p0 + j) * 64)[g] = zb;
      const __nv_bfloat162* zh = reinterpret_cast<const __nv_bfloat162*>(&zb);
      float av[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 zf = __bfloat1622float2(zh[i]);  // the stored pre-activation
        av[2 * i] = gelu(zf.x);
        av[2 * i + 1] = gelu(zf.y);
      }
      put8(a_pad, H, W, c.b, c.y, c.x0 + j, g, pack8(av));
    }
  }
}

// Last layer forward: y = out_scale (conv3x3(a; w[9][64]) + b) (64 -> 1), FP32.
__global__ void __launch_bounds__(kWarps * 32) k_conv_out(int B, int H, int W, float out_scale,
                                                          const __nv_bfloat16* __restrict__ a_pad,
                                                          const float* __restrict__ w, const float* __restrict__ bias,
                                                          float* __restrict__ y) {
  pdl_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float w0[9], w1[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    w0[t] = w[t * 64 + 2 * lane];
    w1[t] = w[t * 64 + 2 * lane + 1];
  }
  const float bb = bias[0];
  const size_t n_chunks = (size_t)B * H * W / kChunk;
  for (size_t ch = (size_t)blockIdx.x * kWarps + warp; ch < n_chunks; ch += (size_t)gridDim.x * kWarps) {
    const Chunk c = chunk_of(ch, H, W);
    float acc[kChunk];
#pragma unroll
    for (int j = 0; j < kChunk; ++j) {
      float s = 0.f;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const float2 f = ld2(a_pad, padidx(c.b, c.y + t / 3 - 1, c.x0 + j + t % 3 - 1, H, W), lane);
        s += f.x * w0[t] + f.y * w1[t];
      }
      acc[j] = s;
    }
    const float tot = reduce_scatter32(acc, lane);
    y[c.p0 + lane] = (tot + bb) * out_scale;
  }
}

// Last layer backward, data part: g_a[q][c] = sum_t gy[q - off_t] w[t][c],
// times gelu'(z[q][c]) -> halo'd BF16 gradient of the layer-5 pre-activation.
__global__ void __launch_bounds__(kWarps * 32) k_conv_out_dgrad(int B, int H, int W, const float* __restrict__ gy,
                                                                const float* __restrict__ w,
                                                                const __nv_bfloat16* __restrict__ z,
                                                                __nv_bfloat16* __restrict__ gz_pad) {
  __shared__ float stg[kWarps][3][34];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float w0[9], w1[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    w0[t] = w[t * 64 + 2 * lane];
    w1[t] = w[t * 64 + 2 * lane + 1];
  }
  const size_t n_chunks = (size_t)B * H * W / kChunk;
  for (size_t ch = (size_t)blockIdx.x * kWarps + warp; ch < n_chunks; ch += (size_t)gridDim.x * kWarps) {
    const Chunk c = chunk_of(ch, H, W);
    __syncwarp();
    stage_rows(stg[warp], gy, H, W, c, lane);
    for (int j = 0; j < kChunk; ++j) {
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int t = 0; t < 9; ++t) {  // gy at (y - dy, x - dx)
        const float g = stg[warp][2 - t / 3][j + 2 - t % 3];
        s0 += g * w0[t];
        s1 += g * w1[t];
      }
      const float2 zz = ld2(z, c.p0 + j, lane);
      put2(gz_pad, H, W, c.b, c.y, c.x0 + j, lane, __floats2bfloat162_rn(s0 * gelu_grad(zz.x), s1 * gelu_grad(zz.y)));
    }
  }
}

// Per-block partial sums of the small-layer gradients (fixed grid, fixed order).
//  mode 0 (last layer):  part[blk][t*64 + c] = sum_p gy[p] a[p + t][c]; part[blk][576] = sum gy
//  mode 1 (first layer): part[blk][t*64 + c] = sum_p gz[p][c] x[p + t];  part[blk][576 + c] = sum gz[.][c]
//  mode 2 (bias of a middle layer): part[blk][576 + c] = sum_p gz[p][c]
constexpr int kRedBlocks = 296;
constexpr int kRedStride = 9 * 64 + 64;
__global__ void __launch_bounds__(kWarps * 32) k_small_grad_partial(int mode, int B, int H, int W,
                                                                    const float* __restrict__ gy,
                                                                    const __nv_bfloat16* __restrict__ a_pad,
                                                                    const float* __restrict__ x,
                                                                    const __nv_bfloat16* __restrict__ gz_pad,
                                                                    float* __restrict__ part) {
  __shared__ float acc[kRedStride];
  __shared__ float stg[kWarps][3][34];
  for (int i = threadIdx.x; i < kRedStride; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float a0[9], a1[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) a0[t] = a1[t] = 0.f;
  float s0 = 0.f, s1 = 0.f;
  const size_t n_chunks = (size_t)B * H * W / kChunk;
  for (size_t ch = (size_t)blockIdx.x * kWarps + warp; ch < n_chunks; ch += (size_t)gridDim.x * kWarps) {
    const Chunk c = chunk_of(ch, H, W);
    if (mode == 0) {
      const float gv = gy[c.p0 + lane];
      s0 += gv;
      for (int j = 0; j < kChunk; ++j) {
        const float g = __shfl_sync(0xffffffffu, gv, j);
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          const float2 f = ld2(a_pad, padidx(c.b, c.y + t / 3 - 1, c.x0 + j + t % 3 - 1, H, W), lane);
          a0[t] += g * f.x;
          a1[t] += g * f.y;
        }
      }
    } else if (mode == 1) {
      __syncwarp();
      stage_rows(stg[warp], x, H, W, c, lane);
      for (int j = 0; j < kChunk; ++j) {
        const float2 g = ld2(gz_pad, padidx(c.b, c.y, c.x0 + j, H, W), lane);
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          const float xv = stg[warp][t / 3][j + t % 3];
          a0[t] += g.x * xv;
          a1[t] += g.y * xv;
        }
        s0 += g.x;
        s1 += g.y;
      }
    } else {
      for (int j = 0; j < kChunk; ++j) {
        const float2 g = ld2(gz_pad, padidx(c.b, c.y, c.x0 + j, H, W), lane);
        s0 += g.x;
        s1 += g.y;
      }
    }
  }
  if (mode == 0) {  // sum of gy over the warp's pixels (fixed order)
    for (int o = 16; o >= 1; o >>= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, o);
  }
  // fixed-order combination of the block's warps
  for (int wv = 0; wv < kWarps; ++wv) {
    if (warp == wv) {
      if (mode != 2) {
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          acc[t * 64 + 2 * lane] += a0[t];
          acc[t * 64 + 2 * lane + 1] += a1[t];
        }
      }
      if (mode == 0) {
        if (lane == 0) acc[576] += s0;
      } else {
        acc[576 + 2 * lane] += s0;
        acc[576 + 2 * lane + 1] += s1;
      }
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

bool shape_ok(int B, int H, int W) { return B >= 1 && H >= 2 && W >= kChunk && W % kChunk == 0; }

// Chunked kernels: enough blocks for every SM several times over, no more
// blocks than there are chunks to share.
int grid_for(int B, int H, int W) {
  const size_t blocks = ((size_t)B * H * W / kChunk + kWarps - 1) / kWarps;
  return (int)(blocks < 1184 ? blocks : 1184);
}

}  // namespace

extern "C" {

int closure_conv_in(int32_t B, int32_t H, int32_t W, float in_scale, const float* x, const float* w, const float* bias,
                    void* z, void* a_pad, void* stream) {
  if (!x || !w || !bias || !z || !a_pad) return ofail("closure_conv_in: null pointer");
  if (!shape_ok(B, H, W)) return ofail("closure_conv_in: need B >= 1, H >= 2 and W a positive multiple of 32");
  const cudaError_t e = launch_pdl(k_conv_in, grid_for(B, H, W), dim3(kWarps * 32), 0, (cudaStream_t)stream, B, H, W,
                                   in_scale, x, w, bias, (__nv_bfloat16*)z, (__nv_bfloat16*)a_pad);
  return e == cudaSuccess ? 0 : ofail("closure_conv_in: launch failed");
}

int closure_conv_out(int32_t B, int32_t H, int32_t W, float out_scale, const void* a_pad, const float* w,
                     const float* bias, float* y, void* stream) {
  if (!a_pad || !w || !bias || !y) return ofail("closure_conv_out: null pointer");
  if (!shape_ok(B, H, W)) return ofail("closure_conv_out: need B >= 1, H >= 2 and W a positive multiple of 32");
  const cudaError_t e = launch_pdl(k_conv_out, grid_for(B, H, W), dim3(kWarps * 32), 0, (cudaStream_t)stream, B, H, W,
                                   out_scale, (const __nv_bfloat16*)a_pad, w, bias, y);
  return e == cudaSuccess ? 0 : ofail("closure_conv_out: launch failed");
}

int closure_conv_out_dgrad(int32_t B, int32_t H, int32_t W, const float* gy, const float* w, const void* z,
                           void* gz_pad, void* stream) {
  if (!gy || !w || !z || !gz_pad) return ofail("closure_conv_out_dgrad: null pointer");
  if (!shape_ok(B, H, W)) return ofail("closure_conv_out_dgrad: need B >= 1, H >= 2 and W a positive multiple of 32");
  k_conv_out_dgrad<<<grid_for(B, H, W), kWarps * 32, 0, (cudaStream_t)stream>>>(B, H, W, gy, w,
                                                                                (const __nv_bfloat16*)z,
                                                                                (__nv_bfloat16*)gz_pad);
  return cudaGetLastError() == cudaSuccess ? 0 : ofail("closure_conv_out_dgrad: launch failed");
}

int closure_small_grad(int32_t mode, int32_t B, int32_t H, int32_t W, const float* gy, const void* a_pad,
                       const float* x, const void* gz_pad, float* partials, float* out, void* stream) {
  if (!partials || !out) return ofail("closure_small_grad: null pointer");
  if (!shape_ok(B, H, W)) return ofail("closure_small_grad: need B >= 1, H >= 2 and W a positive multiple of 32");
  if (mode < 0 || mode > 2) return ofail("closure_small_grad: mode must be 0, 1 or 2");
  if ((mode == 0 && (!gy || !a_pad)) || (mode == 1 && (!x || !gz_pad)) || (mode == 2 && !gz_pad))
    return ofail("closure_small_grad: null input");
  cudaStream_t st = (cudaStream_t)stream;
  k_small_grad_partial<<<kRedBlocks, kWarps * 32, 0, st>>>(mode, B, H, W, gy, (const __nv_bfloat16*)a_pad, x,
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
