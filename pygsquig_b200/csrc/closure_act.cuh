// closure_act.cuh -- the closure network's activation, shared by its kernels.
//
// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units",
// 2016): gelu(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), with the
// hardware tanh approximation (PTX tanh.approx.f32).  The derivative is the
// exact derivative of that form.
#pragma once

__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr float kGeluA = 0.79788456080286536f;  // sqrt(2 / pi)
constexpr float kGeluB = 0.044715f;

__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(kGeluA * z * (1.0f + kGeluB * z * z));
  return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(kGeluA * z * (1.0f + kGeluB * z2));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluA * (1.0f + 3.0f * kGeluB * z2);
}
