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

// Shared-memory index of element i in an exchange buffer of a radix-R
// transform.  Radix 16, and radix 8 in double precision: one padding slot
// every R elements.  Radix 8 in single precision: the low four bits of i are
// XORed with bits 3..9, i ^ (((i >> 3) ^ (i >> 4) ^ (i >> 6)) & 15), which
// puts the 16 eight-byte accesses of a half-warp in 16 different bank pairs
// for every pattern of the transform (the strided loads, the stride 1, 8, 64
// and 512 stores and the radix-2/4 first pass; with the padding rule these
// took 1.6-1.8 shared-memory wavefronts per ideal one).  It changes only the
// low four bits, so it permutes each aligned block of 16 elements.  Radix 4
// in single precision: i ^ ((i >> 2) & 15), conflict-free for its patterns in
// the same way.  A buffer of N elements occupies spad_size<R>(N) = N + N/R
// slots.
template <int R, typename T> __device__ __forceinline__ int spad(int i) {
  if constexpr (R == 8 && sizeof(T) == 4) return i ^ (((i >> 3) ^ (i >> 4) ^ (i >> 6)) & 15);
  else if constexpr (R == 4 && sizeof(T) == 4) return i ^ ((i >> 2) & 15);
  else return i + (i >> (R == 16 ? 4 : 3));
}
template <int R> __host__ __device__ constexpr int spad_size(int n) { return n + n / R; }

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

// Single precision: the same operations on packed pairs (sm_100's two-lane
// FP32 add, multiply and fused multiply-add issue one instruction for both
// components; each lane rounds as the scalar operation does).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// a * b = a.x (b.x, b.y) + a.y (-b.y, b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}
// a * conj(b) = a.x (b.x, -b.y) + a.y (b.y, b.x)
template <bool CONJ> __device__ __forceinline__ float2 cmul_tw(float2 a, float2 b) {
  if (CONJ)
    return __ffma2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), make_float2(b.x, -b.y)));
  return cmul(a, b);
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

// In-place DFTs with sign DIR of v[o + s*r], r = 0..n-1 (natural order).
template <int DIR, typename T, typename C>
__device__ __forceinline__ void dft8s(C* v, int o, int st) {
  C e0 = v[o], e1 = v[o + 2 * st], e2 = v[o + 4 * st], e3 = v[o + 6 * st];
  C o0 = v[o + st], o1 = v[o + 3 * st], o2 = v[o + 5 * st], o3 = v[o + 7 * st];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  const T r = (T)0.70710678118654752440;  // 1/sqrt(2)
  // t1 = o1 (1 + DIR i)/sqrt2 = (o1 + DIR i o1) r;  t3 = o3 (-1 + DIR i)/sqrt2
  const C t1 = cscale(cadd(o1, mul_i<DIR>(o1)), r);
  C t2 = mul_i<DIR>(o2);
  const C t3 = cscale(csub(mul_i<DIR>(o3), o3), r);
  v[o] = cadd(e0, o0); v[o + 4 * st] = csub(e0, o0);
  v[o + st] = cadd(e1, t1); v[o + 5 * st] = csub(e1, t1);
  v[o + 2 * st] = cadd(e2, t2); v[o + 6 * st] = csub(e2, t2);
  v[o + 3 * st] = cadd(e3, t3); v[o + 7 * st] = csub(e3, t3);
}

// 16-point DFT as 4 x 4: DFT4 over the stride-4 subsequences, twiddles
// exp(DIR 2 pi i k m / 16), DFT4 across, transposed write-back.
template <int DIR, typename T, typename C>
__device__ __forceinline__ void dft16(C (&v)[16]) {
  const T c1 = (T)0.92387953251128675613;  // cos(pi/8)
  const T s1 = (T)0.38268343236508977173;  // sin(pi/8)
  const T h = (T)0.70710678118654752440;   // cos(pi/4)
#pragma unroll
  for (int k = 0; k < 4; ++k) dft4<DIR>(v[k], v[k + 4], v[k + 8], v[k + 12]);
  // v[k + 4 m] now holds X_k[m]; multiply by w16^(k m), w16 = exp(DIR 2 pi i / 16)
  auto rot = [&](C a, T c, T s) {  // a * (c + DIR i s) = a c + (DIR i a) s
    if constexpr (sizeof(T) == 4) {
      return __ffma2_rn(mul_i<DIR>(a), make_float2(s, s), __fmul2_rn(a, make_float2(c, c)));
    } else {
      C r;
      r.x = a.x * c - (T)DIR * a.y * s;
      r.y = a.y * c + (T)DIR * a.x * s;
      return r;
    }
  };
  v[5] = rot(v[5], c1, s1);    // k=1 m=1: w^1
  v[9] = rot(v[9], h, h);      // k=1 m=2: w^2
  v[13] = rot(v[13], s1, c1);  // k=1 m=3: w^3
  v[6] = rot(v[6], h, h);      // k=2 m=1: w^2
  v[10] = mul_i<DIR>(v[10]);   // k=2 m=2: w^4
  v[14] = rot(v[14], -h, h);   // k=2 m=3: w^6
  v[7] = rot(v[7], s1, c1);    // k=3 m=1: w^3
  v[11] = rot(v[11], -h, h);   // k=3 m=2: w^6
  v[15] = rot(v[15], -c1, -s1);  // k=3 m=3: w^9
#pragma unroll
  for (int m = 0; m < 4; ++m) dft4<DIR>(v[4 * m], v[4 * m + 1], v[4 * m + 2], v[4 * m + 3]);
  // v[4 m + n] holds X[m + 4 n]; transpose to natural order
  C t[16];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) t[m + 4 * n] = v[4 * m + n];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// NF independent group FFTs executed together.  v[f]: this thread's R
// values of transform f in strided layout, v[f][m] = x_f[j + m G] with
// G = N/R (in and out).  sbuf + f * bstride: spad_size<R>(N) complex slots of
// shared memory for transform f (indexed through spad<R, T>).  The NF
// transforms share every barrier and every twiddle load, which gives each
// thread NF times the independent work per pass.  All threads of the block
// must call it together (it uses __syncthreads).  The routine begins with a
// barrier before its first write to sbuf; on exit other threads may still be
// reading sbuf, so callers synchronise before writing to it again.  Passes:
// one pass of radix 2^(log2 N mod log2 R) first when log2 N is not a multiple
// of log2 R (each thread then runs R / that radix butterflies), then radix-R
// passes.
template <typename T, int LOG2N, int R, int DIR, int NF>
__device__ __forceinline__ void fft_multi(typename Cplx<T>::type (&v)[NF][R], typename Cplx<T>::type* sbuf,
                                          int bstride, int j, const typename Cplx<T>::type* __restrict__ tw) {
  using C = typename Cplx<T>::type;
  constexpr int LR = R == 16 ? 4 : (R == 8 ? 3 : 2);
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / R;
  constexpr int REM = LOG2N % LR;
  constexpr int NPR = LOG2N / LR;
  constexpr bool INV = DIR > 0;
  static_assert(R == 4 || R == 8 || R == 16, "radix 4, 8 or 16");
  static_assert(LOG2N >= LR, "N >= R");
  // Twiddle root of the first radix pass, requested before any work: each
  // pass's root is loaded one pass ahead so the load's latency (the table is
  // often not L1-resident next to large shared-memory buffers) overlaps the
  // butterflies and exchange of the pass before.
  auto root = [&](int pp, int lpp) -> C { return tw[((j & (pp - 1)) << (LOG2N - lpp - LR)) & (N - 1)]; };
  C w_next = REM != 0 ? root(1 << REM, REM) : C{};
  int p = 1;
  if (REM != 0) {
    constexpr int RP = 1 << REM;
    constexpr int NB = R / RP;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        if constexpr (RP == 2) {
          dft2<DIR>(v[f][q], v[f][q + NB]);
        } else if constexpr (RP == 4) {
          dft4<DIR>(v[f][q], v[f][q + NB], v[f][q + 2 * NB], v[f][q + 3 * NB]);
        } else {
          dft8s<DIR, T>(v[f], q, NB);
        }
      }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int i = j + q * G;  // butterfly index, p = 1 so k = 0
#pragma unroll
        for (int r = 0; r < RP; ++r) sbuf[f * bstride + spad<R, T>(i * RP + r)] = v[f][q + r * NB];
      }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int m = 0; m < R; ++m) v[f][m] = sbuf[f * bstride + spad<R, T>(j + m * G)];
    p = RP;
  }
  // Radix-R passes.  The pass loop is kept rolled so that its code is shared
  // by all passes (the unrolled form overflows the instruction cache).
  int lp = REM;  // log2(p)
#pragma unroll 1
  for (int pass = 0; pass < NPR; ++pass) {
    const int k = j & (p - 1);
    const C w_cur = w_next;
    if (pass + 1 < NPR) w_next = root(p * R, lp + LR);
    if (p > 1) {
      // w^r for r = 1..R-1 from one table load w = exp(-+2 pi i k / (p R)):
      // powers by complex products (at most three chained roundings)
      const C w1 = w_cur;
      C wp[R];
      wp[1] = w1;
      wp[2] = cmul(w1, w1);
      wp[3] = cmul(wp[2], w1);
      if constexpr (R >= 8) {
        wp[4] = cmul(wp[2], wp[2]);
        wp[5] = cmul(wp[4], w1);
        wp[6] = cmul(wp[3], wp[3]);
        wp[7] = cmul(wp[4], wp[3]);
      }
      if constexpr (R == 16) {
        wp[8] = cmul(wp[4], wp[4]);
#pragma unroll
        for (int r = 9; r < 16; ++r) wp[r] = cmul(wp[8], wp[r - 8]);
      }
#pragma unroll
      for (int r = 1; r < R; ++r)
#pragma unroll
        for (int f = 0; f < NF; ++f) v[f][r] = cmul_tw<INV>(v[f][r], wp[r]);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      if constexpr (R == 16) dft16<DIR, T>(v[f]);
      else if constexpr (R == 8) dft8s<DIR, T>(v[f], 0, 1);
      else dft4<DIR>(v[f][0], v[f][1], v[f][2], v[f][3]);
    }
    if (pass != NPR - 1) {
      __syncthreads();
      const int base = (j - k) * R + k;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int r = 0; r < R; ++r) sbuf[f * bstride + spad<R, T>(base + r * p)] = v[f][r];
      __syncthreads();
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int m = 0; m < R; ++m) v[f][m] = sbuf[f * bstride + spad<R, T>(j + m * G)];
    }
    p *= R;
    lp += LR;
  }
}

// One group FFT (see fft_multi).
template <typename T, int LOG2N, int R, int DIR>
__device__ __forceinline__ void fft_group(typename Cplx<T>::type (&v)[R], typename Cplx<T>::type* sbuf, int j,
                                          const typename Cplx<T>::type* __restrict__ tw) {
  using C = typename Cplx<T>::type;
  fft_multi<T, LOG2N, R, DIR, 1>(*reinterpret_cast<C(*)[1][R]>(&v), sbuf, 0, j, tw);
}

}  // namespace sqg
