// sqg_fft.cuh -- complex helpers and the block-level FFT used by every pass.
//
// The FFT is a Stockham auto-sort transform executed by a group of G = N/8
// threads.  Thread j of the group holds the eight values x[j + m*G],
// m = 0..7, in registers ("strided layout") before and after the transform,
// so a pass can read its input straight from coalesced global loads and
// write its output with coalesced stores.  Between radix passes the data is
// exchanged through a shared-memory buffer of N complex values owned by the
// group.  Radix-8 passes; when log2(N) is not a multiple of three the first
// pass has radix 2 or 4 (each thread then runs 4 or 2 butterflies).
// Twiddles come from a table tw[k] = exp(-2 pi i k / N) computed on the host
// in float64 from cos/sin (rounded to float for the float path).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sqg {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

template <typename C> __device__ __forceinline__ C mkc(double x, double y) {
  C r; r.x = x; r.y = y; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b) when CONJ, else a * b
template <bool CONJ, typename C> __device__ __forceinline__ C cmul_tw(C a, C b) {
  C r;
  if (CONJ) { r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; }
  else      { r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; }
  return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by DIR * i   (DIR = +1 inverse sign, -1 forward sign)
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
  C r;
  if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

template <int DIR, typename C>
__device__ __forceinline__ void dft2(C& a0, C& a1) {
  C t = a0; a0 = cadd(t, a1); a1 = csub(t, a1);
}

template <int DIR, typename C>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C s02 = cadd(a0, a2), d02 = csub(a0, a2);
  C s13 = cadd(a1, a3), d13 = mul_i<DIR>(csub(a1, a3));
  a0 = cadd(s02, s13); a2 = csub(s02, s13);
  a1 = cadd(d02, d13); a3 = csub(d02, d13);
}

// In-place 8-point DFT with sign DIR of v[0..7] (natural order in and out).
template <int DIR, typename T, typename C>
__device__ __forceinline__ void dft8(C (&v)[8]) {
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  const T r = (T)0.70710678118654752440;  // 1/sqrt(2)
  C t1, t3;
  // o1 * (1 + DIR i)/sqrt2
  t1.x = (o1.x - (T)DIR * o1.y) * r; t1.y = (o1.y + (T)DIR * o1.x) * r;
  C t2 = mul_i<DIR>(o2);
  // o3 * (-1 + DIR i)/sqrt2
  t3.x = (-o3.x - (T)DIR * o3.y) * r; t3.y = (-o3.y + (T)DIR * o3.x) * r;
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
}

// Group FFT.  v: this thread's eight values in strided layout (in and out).
// sbuf: N complex values of shared memory private to the group.  All
// threads of the block must call it together (it uses __syncthreads).
// On entry sbuf may still be read by other threads of the block only if the
// caller synchronises first; the routine begins with a barrier before its
// first write.  On exit other threads may still be reading sbuf: callers
// synchronise before writing to it again.
template <typename T, int LOG2N, int DIR>
__device__ __forceinline__ void fft_group(typename Cplx<T>::type (&v)[8],
                                          typename Cplx<T>::type* sbuf, int j,
                                          const typename Cplx<T>::type* __restrict__ tw) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / 8;
  constexpr int REM = LOG2N % 3;
  constexpr int NP8 = LOG2N / 3;
  constexpr bool INV = DIR > 0;
  static_assert(LOG2N >= 3, "N >= 8");
  int p = 1;
  if (REM != 0) {
    constexpr int RP = 1 << REM;
    constexpr int NB = 8 / RP;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      if (RP == 2) {
        dft2<DIR>(v[q], v[q + NB]);
      } else {
        dft4<DIR>(v[q], v[q + NB], v[q + 2 * NB], v[q + 3 * NB]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int i = j + q * G;  // butterfly index, p = 1 so k = 0
#pragma unroll
      for (int r = 0; r < RP; ++r) sbuf[i * RP + r] = v[q + r * NB];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = sbuf[j + m * G];
    p = RP;
  }
#pragma unroll
  for (int pass = 0; pass < NP8; ++pass) {
    const int k = j & (p - 1);
    if (p > 1) {
      const int stride = N / (p * 8);
#pragma unroll
      for (int r = 1; r < 8; ++r) {
        const C w = tw[(r * k * stride) & (N - 1)];
        v[r] = cmul_tw<INV>(v[r], w);
      }
    }
    dft8<DIR, T>(v);
    if (pass != NP8 - 1) {
      __syncthreads();
      const int base = (j - k) * 8 + k;
#pragma unroll
      for (int r = 0; r < 8; ++r) sbuf[base + r * p] = v[r];
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 8; ++m) v[m] = sbuf[j + m * G];
    }
    p *= 8;
  }
}

}  // namespace sqg
