// sqg_kernels.cuh -- the row and column passes of the pseudo-spectral
// right-hand side and the fused RK4 stage update.
//
// Data path of one RK4 stage for theta (N x N full spectrum, row-major,
// axis 0 = kx, axis 1 = ky):
//
//   row pass  (k_row, one CTA group per row pair (p, N-p), p = 0..N/2):
//       [stage s > 0] forward DFT along y of jh[p][:]      -> J^(p, ky)
//                     RHS = -dealias * J^ + ring forcing (+ L theta_s)
//                     RK4 / IF-RK4 update of rows p and N-p (acc, theta_{s+1})
//       [next stage]  Hermitian part H of theta_{s+1} (and the anti-Hermitian
//                     part A where the reference's .real makes it matter),
//                     spectral multipliers, inverse DFT along y
//                     -> xh[f][p][:]  for f = u, v, theta_x, theta_y
//   column pass (k_col, one CTA group per column pair (y, y+1)):
//       xh[f][0..N/2][y] completes to a Hermitian column, inverse DFT along x
//       -> u, v, theta_x, theta_y at (x, y); J = u theta_x + v theta_y;
//       forward DFT along x of J -> jh[0..N/2][y]
//
// The reference computes the same quantities with nine full complex 2-D FFTs
// per RHS (pygsquig/core/solver.py:28-58, operators.py:101-130).  Because
// every physical-space use goes through ifft2(.).real, only Hermitian
// projections of the multiplied spectra enter; projecting per element pair
// (k, -k) reproduces the reference exactly, including at the Nyquist row and
// column where a derivative multiplier is not Hermitian-symmetric.
#pragma once
#include "sqg_fft.cuh"

namespace sqg {

// Per-row masks of the wavenumber grid, computed on the host with the
// reference's float64 expressions so that every mask edge matches bit for bit
// (grid.py:100-105, damping.py:35-38, ring_forcing.py:74-75).  Entries are
// limits on |m_y|, the integer mode number along y: mode iy is inside the
// dealiasing mask of row ix when |m_y| <= dmax, inside the drag mask when
// |m_y| <= dragmax.  Ring modes of the row are the iy in [pos_lo, pos_hi]
// and [neg_lo, neg_hi] (empty when lo > hi); their ordinals start at
// row_start.
struct RowTab {
  int dmax, dragmax, pos_lo, pos_hi, neg_lo, neg_hi, row_start, pad;
};

enum FieldMode { FM_THETA = 0, FM_VEL = 1, FM_PHYS1 = 2, FM_SCAL = 3 };
enum RowMode { RM_P1 = 0, RM_STAGE = 1, RM_RHS = 2, RM_SPEC = 3 };
enum AlphaKind { AK_GENERAL = 0, AK_ZERO = 1, AK_ONE = 2, AK_HALF = 3, AK_THREEHALF = 4, AK_TWO = 5, AK_MINUSONE = 6 };
enum StageWrite { SW_NONE = 0, SW_FULL = 1, SW_RING = 2 };

struct KP {
  int N, H;
  const double* k1d;  // float64 wavenumbers fftfreq(N, L/N) * 2 pi
  const void* k1t;    // the same in the plan precision
  const void* tw;     // twiddles exp(-2 pi i k/N), plan precision
  const RowTab* rows;
  double inv_n2;      // 1/N^2
  double alpha;
  int akind;
  int scheme;         // 0 explicit RK4, 1 IF-RK4
  // theta linear operator L = -nu_s k2^(ps/2) - nu_d k2^(pd/2) - mu [drag]
  double nu_s, nu_d, mu;
  int ps, pd;
  double dt;
  // ring forcing
  int n_ring;
  int ring_on;
  const double2* ringF;     // [4][n_ring] forcing of each stage (scaled)
  unsigned int* status;
};

struct RowArgs {
  int rmode, fmode, stage;        // stage 1..4
  int do_p1;                      // compute xh of theta_{s+1} (or of the input)
  int stage_write;                // StageWrite for theta_{s+1}
  const void* th_n;               // theta_n (stage 1 input, theta_n for stages 2,3)
  void* th_out;                   // theta_{n+1} (stage 4)
  void* acc;                      // RK4 accumulator
  const void* st_in;              // theta_s for s > 1
  void* st_out;                   // theta_{s+1}
  const void* extra;              // extra RHS (full spectrum) or null
  const void* jh;                 // (N/2+1) x N: row-wise x-transformed J
  void* xh;                       // nf x (N/2+1) x N
  void* rhs_out;                  // RHS mode output
  double kappa;                   // scalar diffusivity (FM_SCAL)
  const void* src_h;              // scalar source spectrum, rows 0..N/2 (FM_SCAL)
  // mean-gradient source spectra of up to 4 scalars, written from theta_{s+1}
  int n_src;
  void* src_out[4];
  double gx[4], gy[4];
};

__device__ __forceinline__ int mode_abs(int i, int N) { return i <= (N >> 1) ? i : N - i; }

// |k|^-alpha with k = 0 -> 0 (operators.py:134-155)
template <typename T>
__device__ __forceinline__ T inv_frac(T k2, T alpha, int kind) {
  if (!(k2 > (T)0)) return (T)0;
  switch (kind) {
    case AK_ZERO: return (T)1;
    case AK_ONE: return (T)1 / sqrt(k2);
    case AK_HALF: return (T)1 / sqrt(sqrt(k2));
    case AK_THREEHALF: { T k = sqrt(k2); return (T)1 / (k * sqrt(k)); }
    case AK_TWO: return (T)1 / k2;
    case AK_MINUSONE: return sqrt(k2);
    default: return pow(sqrt(k2), -alpha);
  }
}

__device__ __forceinline__ double kpow(double k2, int p) {
  // k2^(p/2) for p in {2, 4, 8}
  double k4 = k2 * k2;
  return p == 2 ? k2 : (p == 4 ? k4 : k4 * k4);
}

template <typename C>
__device__ __forceinline__ bool cfinite(C a) { return isfinite(a.x) && isfinite(a.y); }

// Ring ordinal of (row tab, iy) or -1.
__device__ __forceinline__ int ring_ord(const RowTab& rt, int iy) {
  if (iy >= rt.pos_lo && iy <= rt.pos_hi) return rt.row_start + (iy - rt.pos_lo);
  if (iy >= rt.neg_lo && iy <= rt.neg_hi) {
    int npos = rt.pos_hi >= rt.pos_lo ? rt.pos_hi - rt.pos_lo + 1 : 0;
    return rt.row_start + npos + (iy - rt.neg_lo);
  }
  return -1;
}

// ---------------------------------------------------------------------------
// Row pass
// ---------------------------------------------------------------------------
template <typename T, int LOG2N, int RPC>
__global__ void __launch_bounds__(RPC * ((1 << LOG2N) / 8))
k_row(KP kp, RowArgs a) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / 8;
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  const int grp = threadIdx.x / G;
  const int j = threadIdx.x - grp * G;
  C* hbuf = smem + grp * (2 * N);
  C* wbuf = hbuf + N;
  const int p_raw = blockIdx.x * RPC + grp;
  const bool valid = p_raw <= H;
  const int p = valid ? p_raw : H;
  const int pp = (N - p) & (N - 1);
  const bool pair = (p != 0) && (p != H);
  const C* __restrict__ tw = reinterpret_cast<const C*>(kp.tw);
  const T* __restrict__ k1t = reinterpret_cast<const T*>(kp.k1t);
  const RowTab rt = kp.rows[p];
  const double kxd = kp.k1d[p];
  const T kx = k1t[p];
  const T s_n2 = (T)kp.inv_n2;
  bool bad = false;

  C v[8];   // FFT registers
  C t1[8];  // theta_{s+1} (or theta_in) at e1 = (p, iy)
  C t2[8];  // theta_{s+1} at e2 = (pp, N - iy)

  if (a.rmode == RM_P1) {
    const C* th = reinterpret_cast<const C*>(a.th_n);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int iy = j + m * G;
      const int iyp = (N - iy) & (N - 1);
      t1[m] = th[(size_t)p * N + iy];
      t2[m] = th[(size_t)pp * N + iyp];
    }
  } else {
    // forward DFT along y of the x-transformed Jacobian row p
    const C* jh = reinterpret_cast<const C*>(a.jh);
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = jh[(size_t)p * N + j + m * G];
    fft_group<T, LOG2N, -1>(v, wbuf, j, tw);
    // v[m] = J^(p, iy) ; J^(pp, N - iy) = conj(v[m])
    if (a.rmode == RM_SPEC) {
      // forward transform of a real field: rows p and N - p of its spectrum
      C* out = reinterpret_cast<C*>(a.rhs_out);
      if (valid) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int iy = j + m * G;
          out[(size_t)p * N + iy] = v[m];
          if (pair) out[(size_t)pp * N + ((N - iy) & (N - 1))] = cconj(v[m]);
        }
      }
      return;
    }
    const int s = a.stage;
    const bool scal = a.fmode == FM_SCAL;
    const C* th_n = reinterpret_cast<const C*>(a.th_n);
    const C* st_in = reinterpret_cast<const C*>(s == 1 ? a.th_n : a.st_in);
    C* acc = reinterpret_cast<C*>(a.acc);
    C* st_out = reinterpret_cast<C*>(a.st_out);
    C* th_out = reinterpret_cast<C*>(a.th_out);
    const C* extra = reinterpret_cast<const C*>(a.extra);
    const C* src_h = reinterpret_cast<const C*>(a.src_h);
    const double dt = kp.dt;
    const bool explicit_lin = (kp.scheme == 0);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int iy = j + m * G;
      const int iyp = (N - iy) & (N - 1);
      const size_t e1 = (size_t)p * N + iy;
      const size_t e2 = (size_t)pp * N + iyp;
      const int my = mode_abs(iy, N);
      const double kyd = kp.k1d[iy];
      const double k2d = kxd * kxd + kyd * kyd;
      // diagonal linear operator in float64
      double Ld;
      if (scal) {
        Ld = -a.kappa * k2d;
      } else {
        Ld = -kp.nu_s * kpow(k2d, kp.ps) - kp.nu_d * kpow(k2d, kp.pd);
        if (my <= rt.dragmax) Ld -= kp.mu;
      }
      const T dmask = (my <= rt.dmax) ? (T)1 : (T)0;
      C J1 = v[m];
      C n1 = mkc<C>(-dmask * J1.x, -dmask * J1.y);
      C n2 = mkc<C>(-dmask * J1.x, dmask * J1.y);  // conj
      if (scal && src_h) {
        C sh = src_h[(size_t)p * N + iy];
        n1 = cadd(n1, sh);
        n2 = cadd(n2, cconj(sh));
      }
      int ord1 = -1, ord2 = -1;
      if (!scal && kp.ring_on) {
        ord1 = ring_ord(rt, iy);
        if (ord1 >= 0) {
          const double2 F1 = kp.ringF[(size_t)(s - 1) * kp.n_ring + ord1];
          n1.x += (T)F1.x; n1.y += (T)F1.y;
          if (pair) {
            ord2 = ring_ord(kp.rows[pp], iyp);
            if (ord2 >= 0) {
              const double2 F2 = kp.ringF[(size_t)(s - 1) * kp.n_ring + ord2];
              n2.x += (T)F2.x; n2.y += (T)F2.y;
            }
          }
        }
      }
      if (extra) {
        n1 = cadd(n1, extra[e1]);
        if (pair) n2 = cadd(n2, extra[e2]);
      }
      if (a.rmode == RM_RHS) {
        // core RHS (solver.py:28-58): advection + solver hyperviscosity only
        const C x1 = st_in[e1];
        const T Ls = (T)(-kp.nu_s * kpow(k2d, kp.ps));
        C* out = reinterpret_cast<C*>(a.rhs_out);
        if (valid) out[e1] = cadd(n1, cscale(x1, Ls));
        if (pair) {
          const C x2 = st_in[e2];
          if (valid) out[e2] = cadd(n2, cscale(x2, Ls));
        }
        continue;
      }
      C k1v = n1, k2v = n2;
      C xs1 = mkc<C>(0, 0), xs2 = mkc<C>(0, 0);  // stage input
      if (explicit_lin || s == 1) {
        xs1 = st_in[e1];
        if (pair) xs2 = st_in[e2];
      }
      T E = (T)1, E2 = (T)1;
      if (explicit_lin) {
        const T Lt = (T)Ld;
        k1v = cadd(k1v, cscale(xs1, Lt));
        k2v = cadd(k2v, cscale(xs2, Lt));
      } else {
        const double x = Ld * (0.5 * dt);
        const double Ed = x < -745.0 ? 0.0 : exp(x);
        E = (T)Ed;
        E2 = (T)(Ed * Ed);
      }
      const T tdt = (T)dt;
      C o1, o2 = mkc<C>(0, 0);  // theta_{s+1} (or theta_{n+1})
      if (s == 1) {
        // acc = E^2 (th + dt/6 k) ; th2 = E (th + dt/2 k)
        const C a1 = cscale(cadd(xs1, cscale(k1v, tdt / (T)6)), E2);
        if (valid) acc[e1] = a1;
        o1 = cscale(cadd(xs1, cscale(k1v, tdt * (T)0.5)), E);
        if (pair) {
          const C a2 = cscale(cadd(xs2, cscale(k2v, tdt / (T)6)), E2);
          if (valid) acc[e2] = a2;
          o2 = cscale(cadd(xs2, cscale(k2v, tdt * (T)0.5)), E);
        }
      } else if (s == 2 || s == 3) {
        C a1 = acc[e1];
        a1 = cadd(a1, cscale(k1v, tdt / (T)3 * E));
        if (valid) acc[e1] = a1;
        const C x1 = th_n[e1];
        if (s == 2) o1 = cadd(cscale(x1, E), cscale(k1v, tdt * (T)0.5));   // th3 = E th + dt/2 k
        else        o1 = cadd(cscale(x1, E2), cscale(k1v, tdt * E));       // th4 = E^2 th + dt E k
        if (pair) {
          C a2 = acc[e2];
          a2 = cadd(a2, cscale(k2v, tdt / (T)3 * E));
          if (valid) acc[e2] = a2;
          const C x2 = th_n[e2];
          if (s == 2) o2 = cadd(cscale(x2, E), cscale(k2v, tdt * (T)0.5));
          else        o2 = cadd(cscale(x2, E2), cscale(k2v, tdt * E));
        }
      } else {
        // th_{n+1} = acc + dt/6 k
        o1 = cadd(acc[e1], cscale(k1v, tdt / (T)6));
        if (valid) th_out[e1] = o1;
        if (pair) {
          o2 = cadd(acc[e2], cscale(k2v, tdt / (T)6));
          if (valid) th_out[e2] = o2;
        }
      }
      if (s < 4 && valid) {
        if (a.stage_write == SW_FULL || (a.stage_write == SW_RING && ord1 >= 0)) {
          st_out[e1] = o1;
          if (pair) st_out[e2] = o2;
        }
      }
      bad |= !(cfinite(o1) && cfinite(o2));
      t1[m] = o1;
      t2[m] = o2;
    }
  }
  if (kp.status) {
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(kp.status, 1u);
  }
  if (!a.do_p1) return;

  // Rows 0 and N/2 pair with themselves: e2 = (p, N - iy) is owned by another
  // thread of the group, so its new value is exchanged through shared memory.
  if (a.rmode != RM_P1) {
    __syncthreads();
    if (!pair) {
#pragma unroll
      for (int m = 0; m < 8; ++m) hbuf[j + m * G] = t1[m];
    }
    __syncthreads();
    if (!pair) {
#pragma unroll
      for (int m = 0; m < 8; ++m) t2[m] = hbuf[(N - (j + m * G)) & (N - 1)];
    }
    __syncthreads();
  }

  // ---- inverse transforms along y of the multiplied Hermitian projections ----
  C* xh = reinterpret_cast<C*>(a.xh);
  const size_t fstride = (size_t)(H + 1) * N;
  const bool theta_like = (a.fmode == FM_THETA || a.fmode == FM_VEL);
  const T dkx = (p == H) ? (T)0 : kx;
  const T nkx = (p == H) ? kx : (T)0;
  C a_nyq = mkc<C>(0, 0);
  // first field straight from registers
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int iy = j + m * G;
    const C h = cscale(cadd(t1[m], cconj(t2[m])), (T)0.5);
    const C an = cscale(csub(t1[m], cconj(t2[m])), (T)0.5);
    hbuf[j + m * G] = h;
    if (iy == H) a_nyq = an;
    const T ky = k1t[iy];
    const T dky = (iy == H) ? (T)0 : ky;
    C X;
    if (theta_like) {
      const T k2 = kx * kx + ky * ky;
      const T mm = inv_frac<T>(k2, (T)kp.alpha, kp.akind) * s_n2;
      // v: i m (dkx H + nkx A)
      C q = cadd(cscale(h, dkx), cscale(an, nkx));
      X = mkc<C>(-mm * q.y, mm * q.x);
      if (a.n_src > 0 && valid) {
        // u: -i m (dky H + nky A); S^ = -N^2 (gx X_u + gy X_v)
        const T nky = (iy == H) ? ky : (T)0;
        C qu = cadd(cscale(h, dky), cscale(an, nky));
        C Xu = mkc<C>(mm * qu.y, -mm * qu.x);
        const T n2 = (T)1 / s_n2;
        for (int sidx = 0; sidx < a.n_src; ++sidx) {
          C* so = reinterpret_cast<C*>(a.src_out[sidx]);
          const T gx = (T)a.gx[sidx], gy = (T)a.gy[sidx];
          so[(size_t)p * N + iy] = mkc<C>(-n2 * (gx * Xu.x + gy * X.x), -n2 * (gx * Xu.y + gy * X.y));
        }
      }
    } else if (a.fmode == FM_PHYS1) {
      X = cscale(h, s_n2);
    } else {  // FM_SCAL: s_x = i dkx H
      X = mkc<C>(-dkx * s_n2 * h.y, dkx * s_n2 * h.x);
    }
    v[m] = X;
  }
  const int f_first = theta_like ? 1 : 0;
  fft_group<T, LOG2N, +1>(v, wbuf, j, tw);
  if (valid) {
#pragma unroll
    for (int m = 0; m < 8; ++m) xh[f_first * fstride + (size_t)p * N + j + m * G] = v[m];
  }
  int nf = (a.fmode == FM_THETA) ? 4 : (a.fmode == FM_PHYS1 ? 1 : 2);
  for (int f = 0; f < nf; ++f) {
    if (f == f_first) continue;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int iy = j + m * G;
      const C h = hbuf[j + m * G];
      const T ky = k1t[iy];
      const T dky = (iy == H) ? (T)0 : ky;
      C X;
      if (theta_like && f == 0) {
        const T k2 = kx * kx + ky * ky;
        const T mm = inv_frac<T>(k2, (T)kp.alpha, kp.akind) * s_n2;
        const T nky = (iy == H) ? ky : (T)0;
        C q = cadd(cscale(h, dky), cscale(a_nyq, nky));
        X = mkc<C>(mm * q.y, -mm * q.x);
      } else if ((a.fmode == FM_THETA && f == 2)) {
        X = mkc<C>(-dkx * s_n2 * h.y, dkx * s_n2 * h.x);
      } else {  // theta_y or s_y: i dky H
        X = mkc<C>(-dky * s_n2 * h.y, dky * s_n2 * h.x);
      }
      v[m] = X;
    }
    fft_group<T, LOG2N, +1>(v, wbuf, j, tw);
    if (valid) {
#pragma unroll
      for (int m = 0; m < 8; ++m) xh[f * fstride + (size_t)p * N + j + m * G] = v[m];
    }
  }
}

// ---------------------------------------------------------------------------
// Column pass
// ---------------------------------------------------------------------------
// Device-side control of the ring phases for CUDA-graph replays: the phases
// of step n are base + n * n_ring; the column pass of stage 4 advances ctr.
struct RingCtl {
  const double* base;
  int ctr;
  int pad;
};

enum ColMode { CM_THETA = 0, CM_SCAL = 1, CM_VEL = 2, CM_PHYS1 = 3, CM_FWD = 4 };

struct ColArgs {
  int cmode;
  const void* xh;   // nf x (N/2+1) x N
  void* jh;         // (N/2+1) x N
  const void* uv;   // N x N complex u + i v (CM_SCAL input)
  void* out0;       // CM_VEL: u (real N x N) or uv complex; CM_PHYS1: real field
  void* out1;       // CM_VEL: v (real) ; null -> write complex uv into out0
  const void* in_real;  // CM_FWD: real N x N field
  // ring forcing reduction, run by the extra last CTA
  int ring_cta;
  int stage;
  const void* ring_theta;   // theta_s (full spectrum) the rate is measured on
  const double* phases;     // n_ring phases of this step
  RingCtl* ctl;             // if set, phases = ctl->base + ctl->ctr * n_ring
  const int* ring_pos;      // n_ring flat indices ix*N+iy
  const int* ring_mirror;   // ordinal of -k for each ring mode
  double2* ringF;           // [4][n_ring] out
  double2* ou_state;        // n_ring OU state (tau_f > 0)
  int* ou_init;
  double ring_amp, ring_eps, ou_decay, ou_vf;
  int ring_ou;
  int herm_ord[4];          // ordinals of (0,0),(N/2,0),(0,N/2),(N/2,N/2) or -1
  double* ring_scale_out;   // [4]
};

// Complete a half column of a field pair into shared memory:
// Z(kx) = xa + i xb (kx <= N/2), Z(N - kx) = conj(xa) + i conj(xb).
template <typename T>
__device__ __forceinline__ void col_load_pair(const typename Cplx<T>::type* __restrict__ f, int N, int y0,
                                              int npair, typename Cplx<T>::type* smem) {
  using C = typename Cplx<T>::type;
  const int H = N / 2;
  const int total = (H + 1) * npair;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int kx = idx / npair;
    const int q = idx - kx * npair;
    const int ya = y0 + 2 * q;
    const C xa = f[(size_t)kx * N + ya];
    const C xb = f[(size_t)kx * N + ya + 1];
    C* z = smem + (size_t)q * (2 * N);
    if (kx == 0 || kx == H) {
      z[kx] = mkc<C>(xa.x, xb.x);
    } else {
      z[kx] = mkc<C>(xa.x - xb.y, xa.y + xb.x);
      z[N - kx] = mkc<C>(xa.x + xb.y, -xa.y + xb.x);
    }
  }
}

template <typename T, int LOG2N>
__device__ void ring_reduce(const KP& kp, const ColArgs& a);

template <typename T, int LOG2N, int NP>
__global__ void __launch_bounds__(NP * ((1 << LOG2N) / 8))
k_col(KP kp, ColArgs a) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / 8;
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  if (a.ring_cta && blockIdx.x == gridDim.x - 1) {
    ring_reduce<T, LOG2N>(kp, a);
    return;
  }
  const int grp = threadIdx.x / G;
  const int j = threadIdx.x - grp * G;
  C* bufA = smem + grp * (2 * N);
  C* bufB = bufA + N;
  const int y0 = blockIdx.x * (2 * NP);
  const int ya = y0 + 2 * grp;
  const C* __restrict__ tw = reinterpret_cast<const C*>(kp.tw);
  const C* xh = reinterpret_cast<const C*>(a.xh);
  const size_t fstride = (size_t)(H + 1) * N;
  C v[8];

  if (a.cmode == CM_VEL || a.cmode == CM_PHYS1) {
    const int nf = a.cmode == CM_VEL ? 2 : 1;
    // field 0 -> bufA, field 1 -> bufB
    col_load_pair<T>(xh, N, y0, NP, smem);
    if (nf == 2) col_load_pair<T>(xh + fstride, N, y0, NP, smem + N);
    __syncthreads();
    for (int f = 0; f < nf; ++f) {
      C* b = f == 0 ? bufA : bufB;
#pragma unroll
      for (int m = 0; m < 8; ++m) v[m] = b[j + m * G];
      fft_group<T, LOG2N, +1>(v, b, j, tw);
      // v[m] = f(x, ya) + i f(x, ya+1), x = j + m G
      if (a.cmode == CM_PHYS1 || a.out1) {
        T* o = reinterpret_cast<T*>(f == 0 ? a.out0 : a.out1);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const size_t x = j + m * G;
          o[x * N + ya] = v[m].x;
          o[x * N + ya + 1] = v[m].y;
        }
      } else {
        // complex u + i v output
        T* o = reinterpret_cast<T*>(a.out0);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const size_t x = j + m * G;
          o[2 * (x * N + ya) + f] = v[m].x;
          o[2 * (x * N + ya + 1) + f] = v[m].y;
        }
      }
    }
    return;
  }

  // CM_THETA: rounds (u, theta_x), (v, theta_y); CM_SCAL: one round (s_x, s_y)
  C W[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) W[m] = mkc<C>(0, 0);
  if (a.cmode == CM_FWD) {
    const T* f = reinterpret_cast<const T*>(a.in_real);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const size_t x = j + m * G;
      W[m] = mkc<C>(f[x * N + ya], f[x * N + ya + 1]);
    }
  }
  const int nround = a.cmode == CM_THETA ? 2 : (a.cmode == CM_SCAL ? 1 : 0);
  for (int rd = 0; rd < nround; ++rd) {
    if (rd) __syncthreads();
    const int fa = (a.cmode == CM_THETA) ? (rd == 0 ? 0 : 1) : 0;
    const int fb = (a.cmode == CM_THETA) ? (rd == 0 ? 2 : 3) : 1;
    col_load_pair<T>(xh + fa * fstride, N, y0, NP, smem);
    col_load_pair<T>(xh + fb * fstride, N, y0, NP, smem + N);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = bufA[j + m * G];
    fft_group<T, LOG2N, +1>(v, bufA, j, tw);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; ++m) bufA[j + m * G] = v[m];  // velocity-like field, own slots
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = bufB[j + m * G];
    fft_group<T, LOG2N, +1>(v, bufB, j, tw);
    if (a.cmode == CM_THETA) {
      // W += (ua * txa) + i (ub * txb)
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const C u = bufA[j + m * G];
        W[m].x += u.x * v[m].x;
        W[m].y += u.y * v[m].y;
      }
    } else {
      // bufA: s_x(a) + i s_x(b); v: s_y(a) + i s_y(b); uv from global
      const C* uv = reinterpret_cast<const C*>(a.uv);
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const size_t x = j + m * G;
        const C sx = bufA[j + m * G];
        const C w0 = uv[x * N + ya];
        const C w1 = uv[x * N + ya + 1];
        W[m].x = w0.x * sx.x + w0.y * v[m].x;
        W[m].y = w1.x * sx.y + w1.y * v[m].y;
      }
    }
  }
  // forward DFT along x of Ja + i Jb
  fft_group<T, LOG2N, -1>(W, bufA, j, tw);
  __syncthreads();
#pragma unroll
  for (int m = 0; m < 8; ++m) bufA[j + m * G] = W[m];
  __syncthreads();
  // split: Ja(kx) = (W(kx) + conj W(-kx))/2, Jb(kx) = -i (W(kx) - conj W(-kx))/2
  C* jh = reinterpret_cast<C*>(a.jh);
  const int total = (H + 1) * NP;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int kx = idx / NP;
    const int q = idx - kx * NP;
    const C* w = smem + (size_t)q * (2 * N);
    const C wk = w[kx];
    const C wm = w[(N - kx) & (N - 1)];
    const C ja = mkc<C>((T)0.5 * (wk.x + wm.x), (T)0.5 * (wk.y - wm.y));
    const C d = mkc<C>(wk.x - wm.x, wk.y + wm.y);
    const C jb = mkc<C>((T)0.5 * d.y, (T)-0.5 * d.x);
    const int y = y0 + 2 * q;
    jh[(size_t)kx * N + y] = ja;
    jh[(size_t)kx * N + y + 1] = jb;
  }
}

// Ring forcing of one stage (ring_forcing.py:119-170): unit phases times the
// amplitude on the ring, optional OU correlation, DC/Nyquist made real, then
// the rescale eps / <theta F> measured on the stage theta.  <theta F> is the
// mean of Re ifft2(theta) * Re ifft2(F); by Parseval it equals
// N^-4 sum_ring Re[Herm(theta)(k) conj Herm(F)(k)].  One CTA, fixed-order
// reduction (deterministic).
template <typename T, int LOG2N>
__device__ void ring_reduce(const KP& kp, const ColArgs& a) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  __shared__ double red[1024];
  __shared__ double s_scale;
  const int n = kp.n_ring;
  const int s = a.stage;
  double2* F = a.ringF + (size_t)(s - 1) * n;
  const double* phases = a.ctl ? a.ctl->base + (size_t)a.ctl->ctr * n : a.phases;
  // 1. raw forcing of this stage
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double sn, cs;
    sincos(phases[i], &sn, &cs);
    double2 f = make_double2(a.ring_amp * cs, a.ring_amp * sn);
    if (a.ring_ou) {
      if (*a.ou_init) {
        double2 o = a.ou_state[i];
        f = make_double2(a.ou_decay * o.x + a.ou_vf * f.x, a.ou_decay * o.y + a.ou_vf * f.y);
      }
      a.ou_state[i] = f;  // the state keeps the value before the DC/Nyquist fix
    }
    F[i] = f;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (a.ring_ou) *a.ou_init = 1;
    if (a.ctl && s == 4) a.ctl->ctr += 1;  // every thread has read this step's phases
    for (int h = 0; h < 4; ++h) {
      const int o = a.herm_ord[h];
      if (o >= 0) F[o].y = 0.0;
    }
  }
  __syncthreads();
  // 2. rate
  const C* th = reinterpret_cast<const C*>(a.ring_theta);
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int pos = a.ring_pos[i];
    const int ix = pos >> LOG2N, iy = pos & (N - 1);
    const int mpos = (((N - ix) & (N - 1)) << LOG2N) | ((N - iy) & (N - 1));
    const C t1 = th[pos], t2 = th[mpos];
    const double hx = 0.5 * ((double)t1.x + (double)t2.x);
    const double hy = 0.5 * ((double)t1.y - (double)t2.y);
    const double2 f1 = F[i], f2 = F[a.ring_mirror[i]];
    const double fx = 0.5 * (f1.x + f2.x);
    const double fy = 0.5 * (f1.y - f2.y);
    acc += hx * fx + hy * fy;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rate = red[0] * kp.inv_n2 * kp.inv_n2;
    const double sc = fabs(rate) > 1e-10 ? a.ring_eps / rate : 1.0;
    s_scale = sc;
    if (a.ring_scale_out) a.ring_scale_out[s - 1] = sc;
  }
  __syncthreads();
  const double sc = s_scale;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 f = F[i];
    F[i] = make_double2(f.x * sc, f.y * sc);
  }
}

}  // namespace sqg

namespace sqg {
__global__ void k_set_ctl(RingCtl* ctl, const double* base) {
  ctl->base = base;
  ctl->ctr = 0;
}
}  // namespace sqg
