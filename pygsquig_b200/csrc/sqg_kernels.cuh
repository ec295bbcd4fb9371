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
#include "pdl.cuh"
#include "sqg_fft.cuh"
#include "sqg_tma.cuh"

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
// Row-pass instances: one that reads its modes from the arguments; the stage
// passes of theta and of the scalars compiled for their modes alone (any
// stage), or for their modes and one stage s = 1..4 (RI_THETA_S1 + s - 1,
// RI_SCAL_S1 + s - 1); the input passes (RM_P1) of theta, of the scalars and
// of the velocity.
enum RowInst {
  RI_ANY = 0, RI_THETA_STAGE = 1, RI_SCAL_STAGE = 2, RI_THETA_S1 = 3, RI_SCAL_S1 = 7,
  RI_THETA_P1 = 11, RI_SCAL_P1 = 12, RI_VEL_P1 = 13
};
__host__ __device__ constexpr int ri_fmode(int ri) {
  return (ri == RI_THETA_STAGE || ri == RI_THETA_P1 || (ri >= RI_THETA_S1 && ri < RI_SCAL_S1)) ? FM_THETA
         : ((ri == RI_SCAL_STAGE || ri == RI_SCAL_P1 || (ri >= RI_SCAL_S1 && ri < RI_SCAL_S1 + 4))
                ? FM_SCAL
                : (ri == RI_VEL_P1 ? FM_VEL : -1));
}
__host__ __device__ constexpr int ri_rmode(int ri) {
  return ri == RI_ANY ? -1 : (ri >= RI_THETA_P1 ? RM_P1 : RM_STAGE);
}
__host__ __device__ constexpr int ri_stage(int ri) {
  return (ri >= RI_THETA_S1 && ri < RI_SCAL_S1) ? ri - RI_THETA_S1 + 1
         : ((ri >= RI_SCAL_S1 && ri < RI_SCAL_S1 + 4) ? ri - RI_SCAL_S1 + 1 : 0);
}
enum AlphaKind { AK_GENERAL = 0, AK_ZERO = 1, AK_ONE = 2, AK_HALF = 3, AK_THREEHALF = 4, AK_TWO = 5, AK_MINUSONE = 6 };
enum StageWrite { SW_NONE = 0, SW_FULL = 1, SW_RING = 2 };

struct KP {
  int N, H;
  const double* k1d;  // float64 wavenumbers fftfreq(N, L/N) * 2 pi
  const void* k1t;    // the same in the plan precision
  double kval;        // 1 / (N dx): fftfreq's scale (the hot kernels compute k from it)
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
  int rpc;                        // row pairs per CTA (0: the compiled maximum RPC)
};

// ---- asynchronous global -> shared copies (cp.async) ----
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPENDING) : "memory"); }

// Resident blocks per SM the register allocation must allow: at most 128
// registers per thread in float, about 168 in double.
template <typename T>
constexpr int min_blocks(int threads) {
  return sizeof(T) == 4 ? (65536 / (threads * 128) > 8 ? 8 : (65536 / (threads * 128) > 0 ? 65536 / (threads * 128) : 1))
                        : (65536 / (threads * 168) > 8 ? 8 : (65536 / (threads * 168) > 0 ? 65536 / (threads * 168) : 1));
}
// Radix-4 passes keep few values per thread, so their blocks are held to 64
// registers a thread in single precision and 128 in double (more resident
// warps than the radix-8 pass at the same size).
template <typename T, int R>
constexpr int min_blocks_r(int threads) {
  constexpr int regs = sizeof(T) == 4 ? 64 : 128;
  return R == 4 ? (65536 / (threads * regs) > 8 ? 8 : (65536 / (threads * regs) > 0 ? 65536 / (threads * regs) : 1))
                : min_blocks<T>(threads);
}

// NFX of a row pass: 4 or 2 fields transformed together from registers; 6 =
// two at a time with theta_{s+1} parked in shared memory (its Hermitian part
// h, or the row itself on the self-paired rows 0 and N/2), so that the
// transforms hold few registers; 0 = no transforms (the last stage of a step).
__host__ __device__ constexpr int nfx_fields(int nfx) { return nfx == 6 ? 2 : nfx; }
__host__ __device__ constexpr bool nfx_park(int nfx) { return nfx == 6; }

// Row-pass blocks: the passes without inverse transforms (NFX = 0) and the
// parked passes (NFX = 6) are held to the radix-4 register budget (64 a
// thread in single precision, 128 in double), so that more of their blocks
// fit than of the passes that transform fields from registers.
template <typename T, int R, int NFX>
constexpr int row_min_blocks(int threads) {
  return (NFX == 0 || nfx_park(NFX)) ? min_blocks_r<T, 4>(threads) : min_blocks_r<T, R>(threads);
}

__device__ __forceinline__ int mode_abs(int i, int N) { return i <= (N >> 1) ? i : N - i; }

// |k|^-alpha with k = 0 -> 0 (operators.py:134-155)
// Wavenumber of index i computed in registers with numpy's operation order
// for fftfreq(N, L/N) * 2 pi, ((m * val) * 2) * pi, so it equals the k1d table
// bit for bit without a global load per element.
__device__ __forceinline__ double wavenumber(const KP& kp, int i) {
  const int m = i <= ((kp.N - 1) >> 1) ? i : i - kp.N;
  return __dmul_rn(__dmul_rn(__dmul_rn((double)m, kp.kval), 2.0), 3.141592653589793116);
}

// The wavenumber in the arithmetic's precision for the spectral
// multipliers: float64 (then rounded) in double; in float, the same product
// in float arithmetic (within an ulp of the rounded float64 value).
template <typename T>
__device__ __forceinline__ T wavenumber_t(const KP& kp, int i) {
  if constexpr (sizeof(T) == 8) {
    return wavenumber(kp, i);
  } else {
    const int m = i <= ((kp.N - 1) >> 1) ? i : i - kp.N;
    return (float)m * (float)(kp.kval * 6.283185307179586232);
  }
}

template <typename T>
__device__ __forceinline__ T inv_frac(T k2, T alpha, int kind) {
  if (!(k2 > (T)0)) return (T)0;
  if constexpr (sizeof(T) == 4) {
    // single precision: the hardware reciprocal square root (about 2 ulp)
    // instead of correctly rounded square roots and divisions
    const float r1 = rsqrtf(k2);  // 1 / |k|
    switch (kind) {
      case AK_ZERO: return 1.f;
      case AK_ONE: return r1;
      case AK_HALF: return rsqrtf(k2 * r1);             // |k|^-1/2
      case AK_THREEHALF: return r1 * rsqrtf(k2 * r1);   // |k|^-3/2
      case AK_TWO: return r1 * r1;
      case AK_MINUSONE: return k2 * r1;
      default: return powf(k2 * r1, -alpha);
    }
  }
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
// Field kinds of the inverse transforms along y: spectrum X of
//   u: -i m (dky H + nky A)   v: i m (dkx H + nkx A)   (m = |k|^-alpha)
//   dx: i dkx H   dy: i dky H   id: H,   all times 1/N^2,
// where H / A are the Hermitian / anti-Hermitian parts of theta at (k, -k),
// dk = k except 0 on the Nyquist index and nk = k only on the Nyquist index
// (the reference's .real projections, operators.py:15-34, 76-97, 101-130).
enum FieldKind { FK_U = 0, FK_V = 1, FK_DX = 2, FK_DY = 3, FK_ID = 4 };

// Field sets a row_fields call transforms together (fixed at compile time, so
// that each element forms only the spectra of its own kinds): u and v; the
// gradient (dx, dy); all four (u, v, dx, dy); the field itself.
enum FieldSet { FS_UV = 0, FS_GRAD = 1, FS_ALL = 2, FS_ID = 3 };
__host__ __device__ constexpr int fs_fields(int fs) { return fs == FS_ALL ? 4 : (fs == FS_ID ? 1 : 2); }
__host__ __device__ constexpr int fs_kind(int fs, int f) {
  return fs == FS_ID ? FK_ID : (fs == FS_GRAD ? FK_DX + f : f);
}

// The fields of set FS of the row pair's mode: form their spectra from
// theta_{s+1} at (p, iy) / (N-p, N-iy), transform them together along y and
// write xh[f0 + f][p][:].
template <typename T, int LOG2N, int R, int FS, typename HA>
__device__ __forceinline__ void row_fields(const KP& kp, const RowArgs& a, HA ha, int f0, int j, int p, bool valid,
                                           typename Cplx<T>::type* wbuf) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N, G = N / R, H = N / 2, XB = spad_size<R>(N);
  constexpr int NF = fs_fields(FS);
  constexpr bool uv = FS == FS_UV || FS == FS_ALL;  // u and v: the multiplier |k|^-alpha
  const C* __restrict__ tw = reinterpret_cast<const C*>(kp.tw);
  const T kx = wavenumber_t<T>(kp, p);
  const T s_n2 = (T)kp.inv_n2;
  const T dkx = (p == H) ? (T)0 : kx;
  const T nkx = (p == H) ? kx : (T)0;
  C V[NF][R];
#pragma unroll
  for (int m = 0; m < R; ++m) {
    const int iy = j + m * G;
    C h, an;
    ha(m, h, an);
    const T ky = wavenumber_t<T>(kp, iy);
    const T dky = (iy == H) ? (T)0 : ky;
    const T nky = (iy == H) ? ky : (T)0;
    T mm = (T)0;
    if constexpr (uv) mm = inv_frac<T>(kx * kx + ky * ky, (T)kp.alpha, kp.akind) * s_n2;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const int kind = fs_kind(FS, f);
      C X;
      if (kind == FK_U) {
        const C q = cadd(cscale(h, dky), cscale(an, nky));
        X = mkc<C>(mm * q.y, -mm * q.x);
      } else if (kind == FK_V) {
        const C q = cadd(cscale(h, dkx), cscale(an, nkx));
        X = mkc<C>(-mm * q.y, mm * q.x);
      } else if (kind == FK_DX) {
        X = mkc<C>(-dkx * s_n2 * h.y, dkx * s_n2 * h.x);
      } else if (kind == FK_DY) {
        X = mkc<C>(-dky * s_n2 * h.y, dky * s_n2 * h.x);
      } else {
        X = cscale(h, s_n2);
      }
      V[f][m] = X;
    }
    if constexpr (uv) {
      if (a.n_src > 0 && valid) {
        // S^ = -N^2 (gx X_u + gy X_v): the mean-gradient scalar sources, from
        // the u and v spectra of this batch
        const T n2 = (T)1 / s_n2;
        for (int sidx = 0; sidx < a.n_src; ++sidx) {
          C* so = reinterpret_cast<C*>(a.src_out[sidx]);
          const T gx = (T)a.gx[sidx], gy = (T)a.gy[sidx];
          so[(size_t)p * N + iy] =
              mkc<C>(-n2 * (gx * V[0][m].x + gy * V[1][m].x), -n2 * (gx * V[0][m].y + gy * V[1][m].y));
        }
      }
    }
  }
  fft_multi<T, LOG2N, R, +1, NF>(V, wbuf, XB, j, tw);
  if (valid) {
    C* xh = reinterpret_cast<C*>(a.xh);
    const size_t fstride = (size_t)(H + 1) * N;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int m = 0; m < R; ++m) xh[(f0 + f) * fstride + (size_t)p * N + j + m * G] = V[f][m];
  }
}

// Row pass.  DEPTH: how many of the R element chunks of a thread (chunk m =
// the elements iy = j + m G) have their theta_n / acc values prefetched with
// cp.async ahead of use; the first DEPTH chunks are requested before the
// forward FFT of the J row, so their latency hides behind it.
template <typename T, int LOG2N, int R, int RPC, int DEPTH, int NFX, int RI = RI_ANY>
__device__ __forceinline__ void row_body(const KP& kp, const RowArgs& a, int tile) {
  // modes fixed by the instance (RI), else read from the arguments
  const int rmode = ri_rmode(RI) >= 0 ? ri_rmode(RI) : a.rmode;
  const int fmode = ri_fmode(RI) >= 0 ? ri_fmode(RI) : a.fmode;
  const int stage = ri_stage(RI) > 0 ? ri_stage(RI) : a.stage;
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / R;
  constexpr int H = N / 2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  const int grp = threadIdx.x / G;
  const int j = threadIdx.x - grp * G;
  constexpr int XB = spad_size<R>(N);  // one exchange buffer
  constexpr int NFT = nfx_fields(NFX);              // fields transformed together
  constexpr int NB = NFX > 0 ? NFT : 1;            // exchange buffers per group
  C* wbuf = smem + (size_t)grp * NB * XB;
  // prefetch staging: DEPTH chunks x 4 slots (theta_n e1/e2, acc e1/e2) x G
  const int rpc = a.rpc > 0 ? a.rpc : RPC;  // launch shape (autotuned), <= RPC
  C* pf = smem + (size_t)rpc * NB * XB + (size_t)grp * (DEPTH * 4 * G);
  static_assert(!nfx_park(NFX) || DEPTH * 4 * G >= N, "the parked passes keep theta_{s+1} in the staging slots");
  const int p_raw = tile * rpc + grp;
  const bool valid = p_raw <= H;
  const int p = valid ? p_raw : H;
  const int pp = (N - p) & (N - 1);
  const bool pair = (p != 0) && (p != H);
  const C* __restrict__ tw = reinterpret_cast<const C*>(kp.tw);
  const RowTab rt = kp.rows[p];
  const double kxd = wavenumber(kp, p);
  const T kx = (T)kxd;
  const T s_n2 = (T)kp.inv_n2;
  bool bad = false;

  C v[R];   // FFT registers
  C t1[R];  // theta_{s+1} (or theta_in) at e1 = (p, iy)
  C t2[R];  // theta_{s+1} at e2 = (pp, N - iy)

  if (rmode == RM_P1) {
    const C* th = reinterpret_cast<const C*>(a.th_n);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      const int iy = j + m * G;
      const int iyp = (N - iy) & (N - 1);
      t1[m] = th[(size_t)p * N + iy];
      t2[m] = th[(size_t)pp * N + iyp];
    }
  } else {
    // stage pass: request this thread's theta_n / acc elements of the first
    // DEPTH chunks (own slots only, so no barrier is needed to consume them)
    const bool pf_th = rmode == RM_STAGE && stage <= 3;
    const bool pf_acc = rmode == RM_STAGE && stage >= 2;
    const C* pth = reinterpret_cast<const C*>(a.th_n);
    const C* pacc = reinterpret_cast<const C*>(a.acc);
    auto issue = [&](int m) {
      const int iy = j + m * G;
      const int iyp = (N - iy) & (N - 1);
      C* slot = pf + (size_t)(m % DEPTH) * 4 * G + j;
      if (pf_th) {
        cp_async_elem(slot, pth + (size_t)p * N + iy, (int)sizeof(C));
        if (pair) cp_async_elem(slot + G, pth + (size_t)pp * N + iyp, (int)sizeof(C));
      }
      if (pf_acc) {
        cp_async_elem(slot + 2 * G, pacc + (size_t)p * N + iy, (int)sizeof(C));
        if (pair) cp_async_elem(slot + 3 * G, pacc + (size_t)pp * N + iyp, (int)sizeof(C));
      }
      cp_async_commit();
    };
#pragma unroll
    for (int m = 0; m < DEPTH; ++m) issue(m);
    // forward DFT along y of the x-transformed Jacobian row p
    const C* jh = reinterpret_cast<const C*>(a.jh);
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = jh[(size_t)p * N + j + m * G];
    fft_group<T, LOG2N, R, -1>(v, wbuf, j, tw);
    // v[m] = J^(p, iy) ; J^(pp, N - iy) = conj(v[m])
    if (rmode == RM_SPEC) {
      // forward transform of a real field: rows p and N - p of its spectrum
      C* out = reinterpret_cast<C*>(a.rhs_out);
      if (valid) {
#pragma unroll
        for (int m = 0; m < R; ++m) {
          const int iy = j + m * G;
          out[(size_t)p * N + iy] = v[m];
          if (pair) out[(size_t)pp * N + ((N - iy) & (N - 1))] = cconj(v[m]);
        }
      }
      return;
    }
    const int s = stage;
    const bool scal = fmode == FM_SCAL;
    const C* st_in = reinterpret_cast<const C*>(s == 1 ? a.th_n : a.st_in);
    C* acc = reinterpret_cast<C*>(a.acc);
    C* st_out = reinterpret_cast<C*>(a.st_out);
    C* th_out = reinterpret_cast<C*>(a.th_out);
    const C* extra = reinterpret_cast<const C*>(a.extra);
    const C* src_h = reinterpret_cast<const C*>(a.src_h);
    const double dt = kp.dt;
    const bool explicit_lin = (kp.scheme == 0);
    // the scalar's source term is read one chunk ahead, ahead of the wait
    // for the chunk's prefetched values, so that its latency overlaps the
    // element updates of the chunk before
    const bool use_src = scal && src_h != nullptr;
    C sh_next = mkc<C>(0, 0);
    if (use_src) sh_next = src_h[(size_t)p * N + j];
#pragma unroll
    for (int m = 0; m < R; ++m) {
      const int iy = j + m * G;
      const int iyp = (N - iy) & (N - 1);
      const size_t e1 = (size_t)p * N + iy;
      const size_t e2 = (size_t)pp * N + iyp;
      const int my = mode_abs(iy, N);
      const C sh = sh_next;
      if (use_src && m + 1 < R) sh_next = src_h[(size_t)p * N + iy + G];
      cp_async_wait<DEPTH - 1>();  // chunk m has landed (groups are issued in order)
      const C* slot = pf + (size_t)(m % DEPTH) * 4 * G + j;
      const double kyd = wavenumber(kp, iy);
      const double k2d = kxd * kxd + kyd * kyd;
      // diagonal linear operator in float64 (the integrating-factor form's
      // last stage, th_{n+1} = acc + dt/6 k, does not use it)
      double Ld = 0.0;
      if (explicit_lin || s < 4) {
        if (scal) {
          Ld = -a.kappa * k2d;
        } else {
          Ld = -kp.nu_s * kpow(k2d, kp.ps) - kp.nu_d * kpow(k2d, kp.pd);
          if (my <= rt.dragmax) Ld -= kp.mu;
        }
      }
      const T dmask = (my <= rt.dmax) ? (T)1 : (T)0;
      C J1 = v[m];
      C n1 = mkc<C>(-dmask * J1.x, -dmask * J1.y);
      C n2 = mkc<C>(-dmask * J1.x, dmask * J1.y);  // conj
      if (use_src) {
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
      if (rmode == RM_RHS) {
        // core RHS (solver.py:28-58): advection + solver hyperviscosity only
        const C x1 = st_in[e1];
        const T Ls = (T)(-kp.nu_s * kpow(k2d, kp.ps));
        C* out = reinterpret_cast<C*>(a.rhs_out);
        if (valid) out[e1] = cadd(n1, cscale(x1, Ls));
        if (pair) {
          const C x2 = st_in[e2];
          if (valid) out[e2] = cadd(n2, cscale(x2, Ls));
        }
        if (m + DEPTH < R) issue(m + DEPTH);
        else cp_async_commit();
        continue;
      }
      C k1v = n1, k2v = n2;
      C xs1 = mkc<C>(0, 0), xs2 = mkc<C>(0, 0);  // stage input
      if (s == 1) {
        xs1 = slot[0];
        if (pair) xs2 = slot[G];
      } else if (explicit_lin) {
        xs1 = st_in[e1];
        if (pair) xs2 = st_in[e2];
      }
      T E = (T)1, E2 = (T)1;
      if (explicit_lin) {
        const T Lt = (T)Ld;
        k1v = cadd(k1v, cscale(xs1, Lt));
        k2v = cadd(k2v, cscale(xs2, Lt));
      } else if (s < 4) {
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
        C a1 = slot[2 * G];
        a1 = cadd(a1, cscale(k1v, tdt / (T)3 * E));
        if (valid) acc[e1] = a1;
        const C x1 = slot[0];
        if (s == 2) o1 = cadd(cscale(x1, E), cscale(k1v, tdt * (T)0.5));   // th3 = E th + dt/2 k
        else        o1 = cadd(cscale(x1, E2), cscale(k1v, tdt * E));       // th4 = E^2 th + dt E k
        if (pair) {
          C a2 = slot[3 * G];
          a2 = cadd(a2, cscale(k2v, tdt / (T)3 * E));
          if (valid) acc[e2] = a2;
          const C x2 = slot[G];
          if (s == 2) o2 = cadd(cscale(x2, E), cscale(k2v, tdt * (T)0.5));
          else        o2 = cadd(cscale(x2, E2), cscale(k2v, tdt * E));
        }
      } else {
        // th_{n+1} = acc + dt/6 k
        o1 = cadd(slot[2 * G], cscale(k1v, tdt / (T)6));
        if (valid) th_out[e1] = o1;
        if (pair) {
          o2 = cadd(slot[3 * G], cscale(k2v, tdt / (T)6));
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
      if (m + DEPTH < R) issue(m + DEPTH);
      else cp_async_commit();  // empty group keeps the in-order accounting
    }
  }
  if (kp.status) {
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(kp.status, 1u);
  }
  // NFX = 0 is the instantiation for stage passes without the inverse
  // transforms (the last stage of a step): compiled without them, it needs
  // few registers and one exchange buffer, so two blocks share an SM.
  if constexpr (NFX == 0) {
    return;
  } else {
  if (!a.do_p1) return;

  // Rows 0 and N/2 pair with themselves: e2 = (p, N - iy) is owned by another
  // thread of the group, so its new value is exchanged through shared memory
  // (the parked passes read it from the parked row instead).
  if (rmode != RM_P1 && !nfx_park(NFX)) {
    __syncthreads();
    if (!pair) {
#pragma unroll
      for (int m = 0; m < R; ++m) wbuf[j + m * G] = t1[m];
    }
    __syncthreads();
    if (!pair) {
#pragma unroll
      for (int m = 0; m < R; ++m) t2[m] = wbuf[(N - (j + m * G)) & (N - 1)];
    }
  }
  // Hermitian and anti-Hermitian parts of theta_{s+1} at (p, iy), h = (t1 +
  // conj t2) / 2 and an = (t1 - conj t2) / 2, for the transforms: from the
  // registers, or -- in the parked passes, which must fit in 64 registers --
  // from this group's prefetch staging slots, free once the update has
  // consumed them.  On the paired rows an enters only at iy = N/2 (through
  // nky; nkx is zero there), so h alone is parked plus that one value.
  C* hs = pf;
  C anH = mkc<C>(0, 0);  // an at iy = N/2 (element m = R/2 of thread 0)
  if constexpr (nfx_park(NFX)) {
    // park h (paired rows) or the row itself (rows 0 and N/2) in this
    // thread's own staging slots j + m G; the self-paired rows then read the
    // mirrored element of another thread, hence the barrier
#pragma unroll
    for (int m = 0; m < R; ++m) hs[j + m * G] = pair ? cscale(cadd(t1[m], cconj(t2[m])), (T)0.5) : t1[m];
    anH = cscale(csub(t1[R / 2], cconj(t2[R / 2])), (T)0.5);
    __syncthreads();
  }
  auto ha_reg = [&](int m, C& h, C& an) {
    h = cscale(cadd(t1[m], cconj(t2[m])), (T)0.5);
    an = cscale(csub(t1[m], cconj(t2[m])), (T)0.5);
  };
  auto ha_smem = [&](int m, C& h, C& an) {
    const int iy = j + m * G;
    if (pair) {  // the anti-Hermitian part enters only at the Nyquist element
      h = hs[iy];
      an = iy == H ? anH : mkc<C>(0, 0);
    } else {
      const C x1 = hs[iy], x2 = hs[(N - iy) & (N - 1)];
      h = cscale(cadd(x1, cconj(x2)), (T)0.5);
      an = cscale(csub(x1, cconj(x2)), (T)0.5);
    }
  };
  // Inverse transforms along y of the multiplied Hermitian projections, NFT
  // fields at a time (row_fields<.., NF> exchanges through NF <= NB buffers;
  // the batch with u and v also writes the mean-gradient sources).
  static_assert(NFT == 2 || NFT == 4, "row passes with transforms take two or four fields at a time");
  auto fields = [&](auto ha) {
    if (fmode == FM_THETA) {
      if constexpr (NFT == 4) {
        row_fields<T, LOG2N, R, FS_ALL>(kp, a, ha, 0, j, p, valid, wbuf);
      } else {
        row_fields<T, LOG2N, R, FS_UV>(kp, a, ha, 0, j, p, valid, wbuf);
        row_fields<T, LOG2N, R, FS_GRAD>(kp, a, ha, 2, j, p, valid, wbuf);
      }
    } else if (fmode == FM_PHYS1) {
      row_fields<T, LOG2N, R, FS_ID>(kp, a, ha, 0, j, p, valid, wbuf);
    } else if (fmode == FM_VEL) {
      row_fields<T, LOG2N, R, FS_UV>(kp, a, ha, 0, j, p, valid, wbuf);
    } else {
      row_fields<T, LOG2N, R, FS_GRAD>(kp, a, ha, 0, j, p, valid, wbuf);
    }
  };
  if constexpr (nfx_park(NFX)) fields(ha_smem);
  else fields(ha_reg);
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

// CM_SCALV: the first scalar stage of an ensemble step, with u and v
// transformed from theta's half spectra (xh fields 0, 1) beside the scalar's
// s_x, s_y (xh2 fields 0, 1); writes u + i v for the later stages (out0, if
// set).  Needs all four field buffers (NBUF = 4).
enum ColMode { CM_THETA = 0, CM_SCAL = 1, CM_VEL = 2, CM_PHYS1 = 3, CM_FWD = 4, CM_SCALV = 5 };

struct ColArgs {
  int cmode;
  const void* xh;   // nf x (N/2+1) x N
  const void* xh2;  // CM_SCALV: the scalar's s_x, s_y half spectra
  void* jh;         // (N/2+1) x N
  const void* uv;   // N x N complex u + i v (CM_SCAL input)
  void* out0;       // CM_VEL: u (real N x N) or uv complex; CM_PHYS1: real field
  void* out1;       // CM_VEL: v (real) ; null -> write complex uv into out0
  const void* in_real;  // CM_FWD: real N x N field; CM_THETA: source subtracted from J (or null)
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
  int np;                   // column pairs per CTA (0: the compiled maximum NP)
  int tma;                  // 1: the half columns of xh arrive as TMA tiles through the
                            // kernel's tensor map (fields 0.. of the map = xh + f (N/2+1) N)
};

// Velocity u + i v of the scalar passes in physical space, stored
// column-pair-major: the complex (u, v) at (x, y) is element
// ((y / 2) N + x) 2 + (y mod 2), so that a column pair's values for one x are
// adjacent and consecutive x are consecutive (coalesced in the column pass).
__device__ __forceinline__ size_t uv_index(int N, int x, int y) {
  return (((size_t)(y >> 1) * N + x) << 1) + (y & 1);
}
__device__ __forceinline__ void store_pair(float2* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void store_pair(double2* p, double2 a, double2 b) { p[0] = a; p[1] = b; }
__device__ __forceinline__ void load_pair(const float2* p, float2& a, float2& b) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  a = make_float2(q.x, q.y);
  b = make_float2(q.z, q.w);
}
__device__ __forceinline__ void load_pair(const double2* p, double2& a, double2& b) { a = p[0]; b = p[1]; }

// Slots of one field buffer of a column group: the raw half columns of the
// pair, interleaved by row -- slot 2 kx = x(kx, ya), slot 2 kx + 1 =
// x(kx, ya + 1) for kx = 0..N/2 -- later reused as the FFT exchange buffer.
// SZ is even, so every buffer starts on a 16-byte boundary; from
// N = kColTmaMinN on (the sizes whose column passes may take their half
// columns as TMA tiles) a multiple of 16 elements, so that every buffer and
// every 256-row box of it starts on a 128-byte boundary.
constexpr int kColTmaMinN = 1024;
template <int N, int R> struct ColBuf {
  static constexpr int SZ0 = (spad_size<R>(N) + 2 + 1) & ~1;
  static constexpr int SZ = N >= kColTmaMinN ? (SZ0 + 15) & ~15 : SZ0;
};

// 16-byte asynchronous global -> shared copy (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Issue the copies of the half columns of field f for every column pair of
// the block into buffer slot `buf` of each group (no registers, no wait).
// A row of a column pair is 2 sizeof(C) contiguous bytes (one 16-byte copy in
// float, two in double).  Copy unit u = (row kx, pair q, part): part fastest,
// then the pair, so consecutive threads read a row's 16 np contiguous bytes
// and write consecutive 16-byte slots (shifts only: np is a power of two).
//
// With a tensor map (tm, field fidx of its stack): rows 0..N/2-1 of each pair
// arrive as np x N/(2 BH) TMA boxes of BH rows, issued by the lanes of warp 0
// after lane 0 has added their bytes to the group's mbarrier phase (the
// group's one arrival comes from col_commit); row N/2 is one cp.async per
// pair and 16 bytes, as before.
template <typename T, int LOG2N, int R, int NP, int NBUF>
__device__ __forceinline__ void col_fetch(const typename Cplx<T>::type* __restrict__ f, int y0, int buf,
                                          typename Cplx<T>::type* smem, int np, const CUtensorMap* tm = nullptr,
                                          int fidx = 0, uint64_t* bar = nullptr) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N, H = N / 2, SZ = ColBuf<N, R>::SZ;
  constexpr int LC = sizeof(C) == 16 ? 1 : 0;  // log2(16-byte copies per row of a pair)
  const int ls = LC + (31 - __clz(np));        // log2(copy units per row)
  unsigned char* zb = reinterpret_cast<unsigned char*>(smem + (size_t)buf * SZ);
  const unsigned char* gb = reinterpret_cast<const unsigned char*>(f + y0);
  if constexpr (N >= kColTmaMinN) {
    if (tm) {
      constexpr int BH = H < 256 ? H : 256;  // rows per box
      constexpr int NB = H / BH;             // boxes per pair
      constexpr uint32_t kBoxBytes = BH * 2 * sizeof(C);
      static_assert((SZ * sizeof(C)) % 128 == 0 && kBoxBytes % 128 == 0, "TMA boxes start on 128-byte boundaries");
      if (threadIdx.x < 32) {
        if (threadIdx.x == 0) tma_bar_expect(bar, (uint32_t)(np * NB) * kBoxBytes);
        __syncwarp();
        tma_proxy_fence();  // the block's earlier use of the buffers comes before the tile writes
        for (int b = threadIdx.x; b < np * NB; b += 32) {
          const int q = b / NB, c = b - q * NB;
          tma_load_3d(zb + ((size_t)q * NBUF * SZ + 2 * BH * c) * sizeof(C), tm, bar,
                      (y0 + 2 * q) * (int)(sizeof(C) / 4), BH * c, fidx);
        }
      }
      // row H: one 16-byte unit (float) or two (double) per pair
      const int units = 1 << ls;
      for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int part = u & ((1 << LC) - 1);
        const int q = u >> LC;
        cp_async16(zb + ((size_t)q * NBUF * SZ + 2 * H) * sizeof(C) + part * 16,
                   gb + ((size_t)H * N + 2 * q) * sizeof(C) + part * 16);
      }
      return;
    }
  }
  const int units = (H + 1) << ls;
  for (int u = threadIdx.x; u < units; u += blockDim.x) {
    const int part = u & ((1 << LC) - 1);
    const int q = (u >> LC) & (np - 1);
    const int kx = u >> ls;
    cp_async16(zb + ((size_t)q * NBUF * SZ + 2 * kx) * sizeof(C) + part * 16,
               gb + ((size_t)kx * N + 2 * q) * sizeof(C) + part * 16);
  }
}

// First-pass load of a packed column pair: Z(x) = xa + i xb completed to a
// Hermitian column (Z(N - kx) = conj xa + i conj xb), from the raw slots.
template <typename T, int LOG2N, int R>
__device__ __forceinline__ void col_first_load(const typename Cplx<T>::type* z, int j,
                                               typename Cplx<T>::type (&v)[R]) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N, H = N / 2, G = N / R;
#pragma unroll
  for (int m = 0; m < R; ++m) {
    const int x = j + m * G;
    const int kx = x <= H ? x : N - x;
    C xa, xb;
    load_pair(z + 2 * kx, xa, xb);
    if (x == 0 || x == H) v[m] = mkc<C>(xa.x, xb.x);
    else if (x < H) v[m] = mkc<C>(xa.x - xb.y, xa.y + xb.x);
    else v[m] = mkc<C>(xa.x + xb.y, -xa.y + xb.x);
  }
}

template <typename T, int LOG2N>
__device__ void ring_reduce(const KP& kp, const ColArgs& a);

// Column pass.  NBUF = 4: all four fields of the column pairs are fetched at
// once (round-2 copies land while round 1 computes); NBUF = 2: two rounds of
// two fields (large N in float64, where four buffers do not fit).
// CMX >= 0: an instance compiled for that column mode alone (the other
// modes' branches fold away); -1: every mode, chosen by a.cmode at run time.
//
// tm (non-null only from N = kColTmaMinN on, never in CM_SCALV): the field
// stack xh as a tensor map; the half columns then arrive as TMA tiles (a
// commit group's tiles complete on mbarrier colbar[g], one phase per group),
// and a wait that runs out sets kStatusTmaTimeout in kp.status.
template <typename T, int LOG2N, int R, int NP, int NBUF, int CMX = -1>
__device__ __forceinline__ void col_body(const KP& kp, const ColArgs& a, int tile, int ntiles,
                                         const CUtensorMap* tm = nullptr) {
  using C = typename Cplx<T>::type;
  constexpr int N = 1 << LOG2N;
  constexpr int G = N / R;
  constexpr int H = N / 2;
  constexpr int SZ = ColBuf<N, R>::SZ;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  const int cmode = CMX >= 0 ? CMX : a.cmode;
  if ((CMX < 0 || CMX == CM_THETA) && a.ring_cta && tile == ntiles - 1) {
    ring_reduce<T, LOG2N>(kp, a);
    return;
  }
  __shared__ uint64_t colbar[2];
  if constexpr (N < kColTmaMinN) tm = nullptr;
  if (cmode == CM_SCALV || (tma_smem_u32(smem_raw) & 127u) != 0u) tm = nullptr;
  if (tm && threadIdx.x == 0) {
    tma_bar_init(&colbar[0]);
    tma_bar_init(&colbar[1]);
    tma_bar_init_fence();
  }
  // a commit group of copies: the cp.async group and, with tiles, the one
  // arrival of mbarrier g's phase
  auto commit = [&](int g) {
    cp_async_commit();
    if (tm && threadIdx.x == 0) tma_bar_arrive(&colbar[g]);
  };
  // after the cp.async wait and a block barrier: the tiles of group g
  // (after a time-out the flag is set and the thread waits once more, also
  // bounded, since the copies still in flight write this block's buffers;
  // it then carries on, so that no thread leaves the block's barriers)
  auto tile_wait = [&](int g, uint32_t parity) {
    if (tm && !tma_bar_wait(&colbar[g], parity)) {
      if (kp.status) atomicOr(kp.status, kStatusTmaTimeout);
      tma_bar_wait(&colbar[g], parity);
    }
  };
  const int grp = threadIdx.x / G;
  const int j = threadIdx.x - grp * G;
  const int np = a.np > 0 ? a.np : NP;       // launch shape (autotuned), <= NP
  constexpr int qs = NBUF * SZ;              // slots per column pair
  C* gbuf = smem + (size_t)grp * qs;         // this group's NBUF buffers
  const int y0 = tile * (2 * np);
  const int ya = y0 + 2 * grp;
  const C* __restrict__ tw = reinterpret_cast<const C*>(kp.tw);
  const C* xh = reinterpret_cast<const C*>(a.xh);
  const size_t fstride = (size_t)(H + 1) * N;
  C v[R];

  if (cmode == CM_VEL && !a.out1) {
    // u + i v for the scalar passes, column-pair-major (uv_index): both
    // fields transformed together, one 16-byte (float) or two 16-byte
    // (double) stores per thread and row
    col_fetch<T, LOG2N, R, NP, NBUF>(xh, y0, 0, smem, np, tm, 0, &colbar[0]);
    col_fetch<T, LOG2N, R, NP, NBUF>(xh + fstride, y0, 1, smem, np, tm, 1, &colbar[0]);
    commit(0);
    cp_async_wait<0>();
    __syncthreads();
    tile_wait(0, 0);
    C V[2][R];
    col_first_load<T, LOG2N, R>(gbuf, j, V[0]);
    col_first_load<T, LOG2N, R>(gbuf + SZ, j, V[1]);
    fft_multi<T, LOG2N, R, +1, 2>(V, gbuf, SZ, j, tw);
    C* o = reinterpret_cast<C*>(a.out0);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      const int x = j + m * G;
      // V[f][m] = f(x, ya) + i f(x, ya + 1) for f = u, v
      store_pair(o + uv_index(N, x, ya), mkc<C>(V[0][m].x, V[1][m].x), mkc<C>(V[0][m].y, V[1][m].y));
    }
    return;
  }
  if (cmode == CM_VEL || cmode == CM_PHYS1) {
    const int nf = cmode == CM_VEL ? 2 : 1;
    for (int f = 0; f < nf; ++f) col_fetch<T, LOG2N, R, NP, NBUF>(xh + f * fstride, y0, f, smem, np, tm, f, &colbar[0]);
    commit(0);
    cp_async_wait<0>();
    __syncthreads();
    tile_wait(0, 0);
    for (int f = 0; f < nf; ++f) {
      C* b = gbuf + f * SZ;
      col_first_load<T, LOG2N, R>(b, j, v);
      fft_group<T, LOG2N, R, +1>(v, b, j, tw);
      // v[m] = f(x, ya) + i f(x, ya+1), x = j + m G
      if (cmode == CM_PHYS1 || a.out1) {
        T* o = reinterpret_cast<T*>(f == 0 ? a.out0 : a.out1);
#pragma unroll
        for (int m = 0; m < R; ++m) {
          const size_t x = j + m * G;
          o[x * N + ya] = v[m].x;
          o[x * N + ya + 1] = v[m].y;
        }
      } else {
        T* o = reinterpret_cast<T*>(a.out0);  // complex u + i v output
#pragma unroll
        for (int m = 0; m < R; ++m) {
          const size_t x = j + m * G;
          o[2 * (x * N + ya) + f] = v[m].x;
          o[2 * (x * N + ya + 1) + f] = v[m].y;
        }
      }
    }
    return;
  }

  // CM_THETA: the four fields (u, theta_x, v, theta_y) transformed together
  // (NBUF = 4) or in two rounds of two (NBUF = 2); CM_SCAL: one round
  // (s_x, s_y) with (u, v) read from global; CM_FWD: forward transform only.
  C W[R];
#pragma unroll
  for (int m = 0; m < R; ++m) W[m] = mkc<C>(0, 0);
  if (NBUF != 4 && cmode == CM_SCALV) return;  // not supported (the host never asks for it)
  const int nround = (cmode == CM_THETA || cmode == CM_SCALV) ? 2 : (cmode == CM_SCAL ? 1 : 0);
  const int fa0 = 0, fb0 = cmode == CM_THETA ? 2 : 1, fa1 = 1, fb1 = 3;
  if (nround > 0) {
    // CM_SCALV: buffers (u, s_x, v, s_y) -- u, v from theta's xh, s_x, s_y from xh2
    const C* xb = cmode == CM_SCALV ? reinterpret_cast<const C*>(a.xh2) : xh;
    const int fb0s = cmode == CM_SCALV ? 0 : fb0, fb1s = cmode == CM_SCALV ? 1 : fb1;
    // (tm is null in CM_SCALV, so the tile fields are always fields of xh)
    col_fetch<T, LOG2N, R, NP, NBUF>(xh + fa0 * fstride, y0, 0, smem, np, tm, fa0, &colbar[0]);
    col_fetch<T, LOG2N, R, NP, NBUF>(xb + fb0s * fstride, y0, 1, smem, np, tm, fb0s, &colbar[0]);
    if (NBUF == 4 && nround == 2) {
      col_fetch<T, LOG2N, R, NP, NBUF>(xh + fa1 * fstride, y0, 2, smem, np, tm, fa1, &colbar[0]);
      col_fetch<T, LOG2N, R, NP, NBUF>(xb + fb1s * fstride, y0, 3, smem, np, tm, fb1s, &colbar[0]);
    }
    commit(0);
    if (NBUF == 3 && nround == 2) {  // round 2's first field lands in the third buffer during round 1
      col_fetch<T, LOG2N, R, NP, NBUF>(xh + fa1 * fstride, y0, 2, smem, np, tm, fa1, &colbar[1]);
      commit(1);
    }
  }
  if (cmode == CM_FWD) {
    const T* f = reinterpret_cast<const T*>(a.in_real);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      const size_t x = j + m * G;
      W[m] = mkc<C>(f[x * N + ya], f[x * N + ya + 1]);
    }
  }
  if (NBUF == 4 && nround == 2) {
    cp_async_wait<0>();
    __syncthreads();
    tile_wait(0, 0);
    C V[4][R];
#pragma unroll
    for (int f = 0; f < 4; ++f) col_first_load<T, LOG2N, R>(gbuf + f * SZ, j, V[f]);
    fft_multi<T, LOG2N, R, +1, 4>(V, gbuf, SZ, j, tw);
    // J = u theta_x + v theta_y for columns a (real parts) and b (imaginary)
    // (CM_SCALV: u s_x + v s_y)
#pragma unroll
    for (int m = 0; m < R; ++m) {
      W[m].x = V[0][m].x * V[1][m].x + V[2][m].x * V[3][m].x;
      W[m].y = V[0][m].y * V[1][m].y + V[2][m].y * V[3][m].y;
    }
    if (cmode == CM_SCALV && a.out0) {  // u + i v for the later stages (column-pair-major)
      C* o = reinterpret_cast<C*>(a.out0);
#pragma unroll
      for (int m = 0; m < R; ++m)
        store_pair(o + uv_index(N, j + m * G, ya), mkc<C>(V[0][m].x, V[2][m].x), mkc<C>(V[0][m].y, V[2][m].y));
    }
    if (a.in_real) {  // physical-space source: J - src
      const T* f = reinterpret_cast<const T*>(a.in_real);
#pragma unroll
      for (int m = 0; m < R; ++m) {
        const size_t x = j + m * G;
        W[m].x -= f[x * N + ya];
        W[m].y -= f[x * N + ya + 1];
      }
    }
  } else {
    for (int rd = 0; rd < nround; ++rd) {
      if (rd == 1) {
        __syncthreads();  // round-1 buffers free
        if (NBUF != 3) col_fetch<T, LOG2N, R, NP, NBUF>(xh + fa1 * fstride, y0, 0, smem, np, tm, fa1, &colbar[0]);
        col_fetch<T, LOG2N, R, NP, NBUF>(xh + fb1 * fstride, y0, NBUF == 3 ? 0 : 1, smem, np, tm, fb1, &colbar[0]);
        commit(0);  // the second phase of mbarrier 0
      }
      if (NBUF == 3 && rd == 0 && nround == 2) cp_async_wait<1>();  // the third buffer's copies may still fly
      else cp_async_wait<0>();
      __syncthreads();
      tile_wait(0, (uint32_t)rd);
      if (NBUF == 3 && rd == 1) tile_wait(1, 0);
      C V[2][R];
      // buffers of the round's two fields; the transforms exchange through
      // buffers 0 and 1 (fft_multi synchronises before its first write)
      const C* b0 = (NBUF == 3 && rd == 1) ? gbuf + 2 * SZ : gbuf;
      const C* b1 = (NBUF == 3 && rd == 1) ? gbuf : gbuf + SZ;
      col_first_load<T, LOG2N, R>(b0, j, V[0]);
      col_first_load<T, LOG2N, R>(b1, j, V[1]);
      fft_multi<T, LOG2N, R, +1, 2>(V, gbuf, SZ, j, tw);
      if (cmode == CM_THETA) {
#pragma unroll
        for (int m = 0; m < R; ++m) {
          W[m].x += V[0][m].x * V[1][m].x;
          W[m].y += V[0][m].y * V[1][m].y;
        }
      } else {
        // V0: s_x(a) + i s_x(b); V1: s_y(a) + i s_y(b); (u, v) from global
        // (column-pair-major: one coalesced 16-byte load per row in float)
        const C* uvp = reinterpret_cast<const C*>(a.uv);
#pragma unroll
        for (int m = 0; m < R; ++m) {
          const int x = j + m * G;
          C w0, w1;
          load_pair(uvp + uv_index(N, x, ya), w0, w1);
          W[m].x = w0.x * V[0][m].x + w0.y * V[1][m].x;
          W[m].y = w1.x * V[0][m].y + w1.y * V[1][m].y;
        }
      }
    }
  }
  if (!(NBUF == 4 && nround == 2) && cmode == CM_THETA && a.in_real) {  // physical-space source: J - src
    const T* f = reinterpret_cast<const T*>(a.in_real);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      const size_t x = j + m * G;
      W[m].x -= f[x * N + ya];
      W[m].y -= f[x * N + ya + 1];
    }
  }
  // forward DFT along x of Ja + i Jb
  C* bufX = gbuf;
  fft_group<T, LOG2N, R, -1>(W, bufX, j, tw);
  __syncthreads();
#pragma unroll
  for (int m = 0; m < R; ++m) bufX[spad<R, T>(j + m * G)] = W[m];
  __syncthreads();
  // split: Ja(kx) = (W(kx) + conj W(-kx))/2, Jb(kx) = -i (W(kx) - conj W(-kx))/2
  C* jh = reinterpret_cast<C*>(a.jh);
  const int lnp = 31 - __clz(np);  // np is a power of two
  const int total = (H + 1) << lnp;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int kx = idx >> lnp;
    const int q = idx & (np - 1);
    const C* w = smem + (size_t)q * qs;
    const C wk = w[spad<R, T>(kx)];
    const C wm = w[spad<R, T>((N - kx) & (N - 1))];
    const C ja = mkc<C>((T)0.5 * (wk.x + wm.x), (T)0.5 * (wk.y - wm.y));
    const C d = mkc<C>(wk.x - wm.x, wk.y + wm.y);
    const C jb = mkc<C>((T)0.5 * d.y, (T)-0.5 * d.x);
    store_pair(jh + (size_t)kx * N + y0 + 2 * q, ja, jb);
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
  // 2. rate: 256 fixed summation lanes (lane v sums modes v, v + 256, ...),
  // then a tree over the lanes -- the same order whatever the block size
  constexpr int V = 256;
  const C* th = reinterpret_cast<const C*>(a.ring_theta);
  for (int v = threadIdx.x; v < V; v += blockDim.x) {
    double acc = 0.0;
    for (int i = v; i < n; i += V) {
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
    red[v] = acc;
  }
  __syncthreads();
  for (int w = V / 2; w > 0; w >>= 1) {
    for (int v = threadIdx.x; v < w; v += blockDim.x) red[v] += red[v + w];
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
// ---- kernels: one plan, or a batch of members (member = blockIdx.y) ----
template <typename T, int LOG2N, int R, int RPC, int DEPTH, int NFX, int RI = RI_ANY>
__global__ void __launch_bounds__(RPC * ((1 << LOG2N) / R), row_min_blocks<T, R, NFX>(RPC * ((1 << LOG2N) / R)))
k_row(KP kp, RowArgs a) {
  pdl_wait();
  row_body<T, LOG2N, R, RPC, DEPTH, NFX, RI>(kp, a, blockIdx.x);
}

template <typename T, int LOG2N, int R, int NP, int NBUF, int CMX = -1>
__global__ void __launch_bounds__(NP * ((1 << LOG2N) / R), min_blocks_r<T, R>(NP * ((1 << LOG2N) / R)))
k_col(KP kp, ColArgs a, const __grid_constant__ CUtensorMap tm) {
  pdl_wait();
  col_body<T, LOG2N, R, NP, NBUF, CMX>(kp, a, blockIdx.x, gridDim.x, a.tma ? &tm : nullptr);
}

// Batched forms: the member's parameters come from device arrays; members
// with no work in this pass have a null xh pointer and return at once.
template <typename T, int LOG2N, int R, int RPC, int DEPTH, int NFX>
__global__ void __launch_bounds__(RPC * ((1 << LOG2N) / R), row_min_blocks<T, R, NFX>(RPC * ((1 << LOG2N) / R)))
k_row_batch(const KP* __restrict__ kps, const RowArgs* __restrict__ as) {
  pdl_wait();
  const KP& kp = kps[blockIdx.y];  // read in place (a local copy would be indexed dynamically)
  const RowArgs& a = as[blockIdx.y];
  if (a.xh == nullptr && a.rhs_out == nullptr) return;
  row_body<T, LOG2N, R, RPC, DEPTH, NFX>(kp, a, blockIdx.x);
}

template <typename T, int LOG2N, int R, int NP, int NBUF>
__global__ void __launch_bounds__(NP * ((1 << LOG2N) / R), min_blocks_r<T, R>(NP * ((1 << LOG2N) / R)))
k_col_batch(const KP* __restrict__ kps, const ColArgs* __restrict__ as) {
  pdl_wait();
  const KP& kp = kps[blockIdx.y];
  const ColArgs& a = as[blockIdx.y];
  if (a.xh == nullptr) return;
  col_body<T, LOG2N, R, NP, NBUF>(kp, a, blockIdx.x, gridDim.x);
}
}  // namespace sqg
