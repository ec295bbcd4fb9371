// sqg_aux.cuh -- small kernels around the passes: damping term, ring-forcing
// scatter, float64 diagnostics reductions, max |field|.
#pragma once
#include <math_constants.h>

#include "sqg_kernels.cuh"

namespace sqg {
// Points the graph-replayed ring-phase control block at a phase table.
__global__ void k_set_ctl(RingCtl* ctl, const double* base) {
  ctl->base = base;
  ctl->ctr = 0;
}
}  // namespace sqg

namespace sqg {

// out = L * theta, L = -mu [|k| < kf/2] - nu k2^(p/2): the damping term of
// CombinedDamping.__call__ (damping.py:75-92) or, with mu = 0, the solver's
// hyperviscosity (operators.py:185-207; zero at k = 0 because k2 = 0 there).
template <typename T>
__global__ void k_linear(KP kp, double nu, int pw, double mu, const typename Cplx<T>::type* __restrict__ th,
                         typename Cplx<T>::type* __restrict__ out) {
  using C = typename Cplx<T>::type;
  const int N = kp.N;
  const size_t total = (size_t)N * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(e / N), iy = (int)(e - (size_t)ix * N);
    const double kx = kp.k1d[ix], ky = kp.k1d[iy];
    const double k2 = kx * kx + ky * ky;
    double L = -nu * kpow(k2, pw);
    if (mu != 0.0 && mode_abs(iy, N) <= kp.rows[ix].dragmax) L -= mu;
    out[e] = cscale(th[e], (T)L);
  }
}

// Full forcing spectrum from the scaled ring values of stage 1.
template <typename T>
__global__ void k_ring_scatter(int n_ring, const int* __restrict__ pos, const double2* __restrict__ F,
                               typename Cplx<T>::type* __restrict__ out) {
  using C = typename Cplx<T>::type;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_ring; i += gridDim.x * blockDim.x) {
    out[pos[i]] = mkc<C>(F[i].x, F[i].y);
  }
}

// Block reduction of NV doubles (sum), blockDim.x power of two <= 1024.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sred) {
  for (int q = 0; q < NV; ++q) {
    sred[q * blockDim.x + threadIdx.x] = v[q];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int q = 0; q < NV; ++q) sred[q * blockDim.x + threadIdx.x] += sred[q * blockDim.x + threadIdx.x + w];
    __syncthreads();
  }
  for (int q = 0; q < NV; ++q) v[q] = sred[q * blockDim.x];
  __syncthreads();
}

// Spectral diagnostics partial sums per block (fixed grid -> deterministic):
//  0: sum k2^((a-2)/2) |th|^2 (k != 0)     energy numerator
//  1: sum |k|^(2a) |th|^2                  enstrophy numerator (k=0 -> 0)
//  2: sum |U|^2 + |V|^2                    U, V = fft2 of u, v (Herm projections)
//  3: sum |Herm th|^2                      N^4 <theta^2>
//  4: sum k2^(1+a) |th|^2 (k != 0)         palinstrophy numerator
template <typename T>
__global__ void k_diag_partial(KP kp, const typename Cplx<T>::type* __restrict__ th, double* partial) {
  using C = typename Cplx<T>::type;
  constexpr int NV = 5;
  __shared__ double sred[NV * 256];
  const int N = kp.N, H = N / 2;
  const size_t total = (size_t)N * N;
  double acc[NV] = {0, 0, 0, 0, 0};
  const double a = kp.alpha;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(e / N), iy = (int)(e - (size_t)ix * N);
    const int ixp = (N - ix) & (N - 1), iyp = (N - iy) & (N - 1);
    const C t1 = th[e];
    const C t2 = th[(size_t)ixp * N + iyp];
    const double tx = t1.x, ty = t1.y;
    const double kx = kp.k1d[ix], ky = kp.k1d[iy];
    const double k2 = kx * kx + ky * ky;
    const double a2 = tx * tx + ty * ty;
    const double hx = 0.5 * ((double)t1.x + (double)t2.x), hy = 0.5 * ((double)t1.y - (double)t2.y);
    const double ax = 0.5 * ((double)t1.x - (double)t2.x), ay = 0.5 * ((double)t1.y + (double)t2.y);
    if (k2 > 0) {
      acc[0] += pow(k2, (a - 2.0) / 2.0) * a2;
      acc[1] += pow(sqrt(k2), a) * pow(sqrt(k2), a) * a2;
      acc[4] += pow(k2, 1.0 + a) * a2;
      double m = pow(sqrt(k2), -a);
      const double dkx = ix == H ? 0.0 : kx, nkx = ix == H ? kx : 0.0;
      const double dky = iy == H ? 0.0 : ky, nky = iy == H ? ky : 0.0;
      // U = -i m (dky H + nky A), V = i m (dkx H + nkx A)
      const double ux = m * (dky * hx + nky * ax), uy = m * (dky * hy + nky * ay);
      const double vx = m * (dkx * hx + nkx * ax), vy = m * (dkx * hy + nkx * ay);
      acc[2] += ux * ux + uy * uy + vx * vx + vy * vy;
    } else if (a == 0.0) {
      // (k2 > 0 fails only at k = 0) |k|^0 -> where(k2>0,...,0) = 0
    }
    acc[3] += hx * hx + hy * hy;
  }
  block_sum<NV>(acc, sred);
  if (threadIdx.x == 0)
    for (int q = 0; q < NV; ++q) partial[(size_t)blockIdx.x * NV + q] = acc[q];
}

// Final fixed-order reduction of the partial sums into the diagnostics vector.
__global__ void k_diag_final(int nblocks, int N, const double* partial, const double* maxv, double* out) {
  constexpr int NV = 5;
  __shared__ double sred[NV * 256];
  double acc[NV] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < NV; ++q) acc[q] += partial[(size_t)b * NV + q];
  block_sum<NV>(acc, sred);
  if (threadIdx.x == 0) {
    const double n2 = (double)N * (double)N;
    out[0] = 0.5 * acc[0] / n2;
    out[1] = 0.5 * acc[1];
    out[2] = 0.5 * acc[2] / (n2 * n2);
    out[3] = 0.5 * acc[3] / (n2 * n2);
    out[4] = maxv ? *maxv : 0.0;
    out[5] = 0.5 * acc[4] / n2;
  }
}

// max |f| over a real field: per-block maxima then a final pass.
template <typename T>
__global__ void k_absmax_partial(const T* __restrict__ f, size_t n, double* partial) {
  __shared__ double sm[256];
  double m = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs((double)f[i]));
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void k_absmax_final(int nblocks, const double* partial, double* out) {
  __shared__ double sm[256];
  double m = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = fmax(m, partial[b]);
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

// Shell spectrum partials: per block, n_bins sums of the energy density
// 1/2 |k|^(a-2) |th|^2 (k = 0 excluded) over edges[i] <= |k| < edges[i+1]
// (utils/diagnostics.py:22-84).
template <typename T>
__global__ void k_spectrum_partial(KP kp, const typename Cplx<T>::type* __restrict__ th, const double* edges,
                                   int n_bins, double* partial) {
  using C = typename Cplx<T>::type;
  __shared__ double sb[64];
  for (int i = threadIdx.x; i < 64; i += blockDim.x) sb[i] = 0.0;
  __syncthreads();
  const int N = kp.N;
  const size_t total = (size_t)N * N;
  const double step = edges[1];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(e / N), iy = (int)(e - (size_t)ix * N);
    if (ix == 0 && iy == 0) continue;
    const double kx = kp.k1d[ix], ky = kp.k1d[iy];
    const double km = sqrt(kx * kx + ky * ky);
    int b = (int)floor(km / step);
    if (b > n_bins) b = n_bins;
    while (b > 0 && km < edges[b]) --b;
    while (b < n_bins && km >= edges[b + 1]) ++b;
    if (b >= n_bins) continue;
    const C t = th[e];
    const double ed = 0.5 * pow(km, kp.alpha - 2.0) * ((double)t.x * t.x + (double)t.y * t.y);
    atomicAdd(&sb[b], ed);  // shared-memory partial; order within a block only
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n_bins; i += blockDim.x) partial[(size_t)blockIdx.x * 64 + i] = sb[i];
}

__global__ void k_spectrum_final(int nblocks, int n_bins, const double* partial, const double* edges, double* out) {
  for (int i = threadIdx.x; i < n_bins; i += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * 64 + i];
    out[i] = s / (edges[i + 1] - edges[i]);
  }
}

// Scalar variance <(s - <s>)^2> = N^-4 sum_{k != 0} |Herm s(k)|^2.
template <typename T>
__global__ void k_var_partial(int N, const typename Cplx<T>::type* __restrict__ sh, double* partial) {
  using C = typename Cplx<T>::type;
  __shared__ double sred[256];
  const size_t total = (size_t)N * N;
  double acc[1] = {0.0};
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    if (e == 0) continue;
    const int ix = (int)(e / N), iy = (int)(e - (size_t)ix * N);
    const C t1 = sh[e];
    const C t2 = sh[(size_t)((N - ix) & (N - 1)) * N + ((N - iy) & (N - 1))];
    const double hx = 0.5 * ((double)t1.x + (double)t2.x), hy = 0.5 * ((double)t1.y - (double)t2.y);
    acc[0] += hx * hx + hy * hy;
  }
  block_sum<1>(acc, sred);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

__global__ void k_var_final(int nblocks, int N, const double* partial, double* out) {
  __shared__ double sred[256];
  double acc[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc[0] += partial[b];
  block_sum<1>(acc, sred);
  if (threadIdx.x == 0) {
    const double n2 = (double)N * (double)N;
    *out = acc[0] / (n2 * n2);
  }
}

}  // namespace sqg

namespace sqg {
// <Re ifft2(a) Re ifft2(b)> = N^-4 sum_k Re[Herm a(k) conj Herm b(k)]
template <typename T>
__global__ void k_inner_partial(int N, const typename Cplx<T>::type* __restrict__ a,
                                const typename Cplx<T>::type* __restrict__ b, double* partial) {
  using C = typename Cplx<T>::type;
  __shared__ double sred[256];
  const size_t total = (size_t)N * N;
  double acc[1] = {0.0};
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(e / N), iy = (int)(e - (size_t)ix * N);
    const size_t em = (size_t)((N - ix) & (N - 1)) * N + ((N - iy) & (N - 1));
    const C a1 = a[e], a2 = a[em], b1 = b[e], b2 = b[em];
    const double hax = 0.5 * ((double)a1.x + (double)a2.x), hay = 0.5 * ((double)a1.y - (double)a2.y);
    const double hbx = 0.5 * ((double)b1.x + (double)b2.x), hby = 0.5 * ((double)b1.y - (double)b2.y);
    acc[0] += hax * hbx + hay * hby;
  }
  block_sum<1>(acc, sred);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}
}  // namespace sqg

namespace sqg {
// Forcing-only RK4 sub-steps on the ring modes (split forcing of a coarse
// solve).  For fixed raw forcing F (amplitude x exp(i phase) on the ring, DC
// and Nyquist entries real) the reference's stage forcing is s(r) F with
// s(r) = eps / r (1 if |r| <= 1e-10) and r = <theta F> (ring_forcing.py:
// 151-170).  r is linear in theta, r(theta + c F) = r(theta) + c Q with
// Q = <F F>, so the RK4 step of d theta/dt = s(r(theta)) F is
//   r1 = r(theta), r2 = r1 + dt/2 s1 Q, r3 = r1 + dt/2 s2 Q, r4 = r1 + dt s3 Q,
//   theta += dt/6 (s1 + 2 s2 + 2 s3 + s4) F.
// <a b> = N^-4 sum_ring Re[Herm a(k) conj Herm b(k)] (Parseval).  One CTA;
// fixed-order 256-lane sums.
template <typename T>
__global__ void __launch_bounds__(256) k_ring_substeps(int N, int n, const int* __restrict__ ring_pos,
                                                       const int* __restrict__ ring_mirror, int4 herm_ord,
                                                       double amp, double eps, int n_sub, double dt,
                                                       const double* __restrict__ phases,
                                                       typename Cplx<T>::type* theta, double2* F) {
  pdl_wait();
  using C = typename Cplx<T>::type;
  constexpr int V = 256;  // launched with exactly V threads
  __shared__ double red_r[V / 32], red_q[V / 32];
  __shared__ double s_c;
  const int ho[4] = {herm_ord.x, herm_ord.y, herm_ord.z, herm_ord.w};
  const double inv_n4 = 1.0 / ((double)N * N * (double)N * N);
  for (int m = 0; m < n_sub; ++m) {
    const double* ph = phases + (size_t)m * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double sn, cs;
      sincos(ph[i], &sn, &cs);
      double fy = amp * sn;
      for (int h = 0; h < 4; ++h)
        if (ho[h] == i) fy = 0.0;
      F[i] = make_double2(amp * cs, fy);
    }
    __syncthreads();
    // fixed-order reduction: each thread sums its strided modes, warps
    // reduce by shuffles, thread 0 adds the eight warp sums in order
    double ar = 0.0, aq = 0.0;
    for (int i = threadIdx.x; i < n; i += V) {
      const int pos = ring_pos[i];
      const int ix = pos / N, iy = pos - ix * N;
      const int mpos = ((N - ix) & (N - 1)) * N + ((N - iy) & (N - 1));
      const C t1 = theta[pos], t2 = theta[mpos];
      const double hx = 0.5 * ((double)t1.x + (double)t2.x);
      const double hy = 0.5 * ((double)t1.y - (double)t2.y);
      const double2 f1 = F[i], f2 = F[ring_mirror[i]];
      const double fx = 0.5 * (f1.x + f2.x), fy = 0.5 * (f1.y - f2.y);
      ar += hx * fx + hy * fy;
      aq += fx * fx + fy * fy;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ar += __shfl_down_sync(0xffffffffu, ar, o);
      aq += __shfl_down_sync(0xffffffffu, aq, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red_r[threadIdx.x >> 5] = ar;
      red_q[threadIdx.x >> 5] = aq;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sr = 0.0, sq = 0.0;
      for (int w = 0; w < V / 32; ++w) {
        sr += red_r[w];
        sq += red_q[w];
      }
      const double r1 = sr * inv_n4, q = sq * inv_n4;
      auto sc = [&](double r) { return fabs(r) > 1e-10 ? eps / r : 1.0; };
      const double s1 = sc(r1);
      const double s2 = sc(r1 + 0.5 * dt * s1 * q);
      const double s3 = sc(r1 + 0.5 * dt * s2 * q);
      const double s4 = sc(r1 + dt * s3 * q);
      s_c = dt / 6.0 * (s1 + 2.0 * s2 + 2.0 * s3 + s4);
    }
    __syncthreads();
    const double c = s_c;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int pos = ring_pos[i];
      const double2 f = F[i];
      C t = theta[pos];
      t.x = (T)((double)t.x + c * f.x);
      t.y = (T)((double)t.y + c * f.y);
      theta[pos] = t;
    }
    __syncthreads();
  }
}
}  // namespace sqg

namespace sqg {
// Maxima for adaptive stepping (adaptive_timestep.py:59-68, 288-305): per
// block, max sqrt(u^2 + v^2) of two real fields, or max |z| of a complex
// field; a non-finite element makes the block's value NaN.  Max is
// order-independent, so the result is deterministic.
template <typename T>
__global__ void k_speedmax_partial(const T* __restrict__ u, const T* __restrict__ v, size_t n, double* partial) {
  __shared__ double sm[256];
  double m = 0.0;
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double a = (double)u[i], b = (double)v[i];
    const double s = sqrt(a * a + b * b);
    bad |= !isfinite(s);
    m = fmax(m, s);
  }
  sm[threadIdx.x] = bad ? CUDART_NAN : m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const double x = sm[threadIdx.x], y = sm[threadIdx.x + w];
      sm[threadIdx.x] = (isnan(x) || isnan(y)) ? CUDART_NAN : fmax(x, y);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}
template <typename C>
__global__ void k_cabsmax_partial(const C* __restrict__ z, size_t n, double* partial) {
  __shared__ double sm[256];
  double m = 0.0;
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double a = (double)z[i].x, b = (double)z[i].y;
    const double s = sqrt(a * a + b * b);
    bad |= !isfinite(s);
    m = fmax(m, s);
  }
  sm[threadIdx.x] = bad ? CUDART_NAN : m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const double x = sm[threadIdx.x], y = sm[threadIdx.x + w];
      sm[threadIdx.x] = (isnan(x) || isnan(y)) ? CUDART_NAN : fmax(x, y);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}
__global__ void k_nanmax_final(int nblocks, const double* partial, double* out) {
  __shared__ double sm[256];
  double m = 0.0;
  bool bad = false;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    bad |= isnan(partial[b]);
    m = fmax(m, partial[b]);
  }
  sm[threadIdx.x] = bad ? CUDART_NAN : m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const double x = sm[threadIdx.x], y = sm[threadIdx.x + w];
      sm[threadIdx.x] = (isnan(x) || isnan(y)) ? CUDART_NAN : fmax(x, y);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}
}  // namespace sqg
