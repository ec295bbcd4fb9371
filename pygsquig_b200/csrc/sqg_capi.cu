// sqg_capi.cu -- plan management, host-side tables and the extern "C" entry
// points declared in include/sqg.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sqg.h"
#include "sqg_aux.cuh"
#include "sqg_launch.cuh"

using namespace sqg;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define SQG_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t err__ = (call);                                                     \
    if (err__ != cudaSuccess)                                                       \
      return fail(SQG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err__)); \
  } while (0)

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct sqg_plan {
  sqg_desc d;
  int N, H, log2N;
  size_t csize;  // bytes per complex element
  int akind;
  // host tables
  std::vector<double> k1d;
  std::vector<RowTab> rows;
  std::vector<int> ring_pos, ring_mirror;
  int herm_ord[4];
  std::vector<double> edges;
  int n_bins;
  double ou_decay, ou_vf;
  // workspace
  unsigned char* ws = nullptr;
  size_t ws_bytes = 0;
  size_t off_k1d, off_k1t, off_tw, off_rows, off_ring_pos, off_ring_mirror, off_ringF, off_ring_scale,
      off_ou_state, off_ou_init, off_status, off_step_ctr, off_acc, off_stage, off_xh, off_jh, off_uv, off_xs, off_js,
      off_sacc, off_sstage, off_src, off_part, off_edges, off_phys, off_state, off_ctl, off_total;
  int n_src_buf;
  bool ready = false;
  bool stage_begun = false;
  int rpc = 0, np = 0;  // launch shapes of the row / column passes (0: compiled maximum)
  int64_t launches = 0;
  // CUDA graph of one steady-state step (multistep)
  cudaGraphExec_t graph_exec = nullptr;
  const void* graph_theta = nullptr;
  const double* graph_phases = nullptr;
  double graph_dt = 0.0;
  cudaStream_t cap_stream = nullptr;  // plan-owned stream the graph is captured on and replayed on
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // TMA tile loads of the column passes (N >= kColTmaMinN): tensor maps of
  // the field stacks xh and xs, encoded when the workspace is bound
  bool col_tma = false;
  CUtensorMap map_xh, map_xs;
  // per-launch CUDA-event timing (bench instrumentation)
  bool timing = false;
  int timing_reps = 1;  // launches per launch site while timing
  std::vector<cudaEvent_t> ev_pool;
  struct Rec { int kind; cudaEvent_t a, b; int reps; };
  std::vector<Rec> recs;
  size_t ev_used = 0;
};

namespace {

constexpr int kPartBlocks = 296;  // 2 x 148 SMs

template <typename P> P* wsp(const sqg_plan* pl, size_t off) { return reinterpret_cast<P*>(pl->ws + off); }

// fftfreq(N, d=L/N) * 2 * pi, evaluated in the order numpy uses so that the
// values are bit-identical to the reference's grid (grid.py:88-95).
std::vector<double> wavenumbers(int N, double L) {
  const double dx = L / N;
  const double val = 1.0 / (N * dx);
  std::vector<double> k(N);
  const int npos = (N - 1) / 2 + 1;
  for (int i = 0; i < N; ++i) {
    const long m = i < npos ? i : (long)i - N;
    k[i] = (((double)m * val) * 2.0) * M_PI;
  }
  return k;
}

int alpha_kind(double a) {
  if (a == 0.0) return AK_ZERO;
  if (a == 1.0) return AK_ONE;
  if (a == 0.5) return AK_HALF;
  if (a == 1.5) return AK_THREEHALF;
  if (a == 2.0) return AK_TWO;
  if (a == -1.0) return AK_MINUSONE;
  return AK_GENERAL;
}

void build_tables(sqg_plan* pl) {
  const int N = pl->N, H = pl->H;
  const sqg_desc& d = pl->d;
  pl->k1d = wavenumbers(N, d.L);
  const std::vector<double>& k = pl->k1d;
  // dealias cutoff (2/3) * pi * N / L, grid.py:102-105
  const double k_max = M_PI * N / d.L;
  const double cutoff = (2.0 / 3.0) * k_max;
  const double drag_half = d.kf_damp / 2;
  const double ring_half = d.ring_dk / 2;
  pl->rows.assign(N, RowTab{});
  pl->ring_pos.clear();
  for (int ix = 0; ix < N; ++ix) {
    RowTab& rt = pl->rows[ix];
    const double kx2 = k[ix] * k[ix];
    rt.dmax = -1;
    rt.dragmax = -1;
    int lo = H + 1, hi = -1;
    for (int my = 0; my <= H; ++my) {
      const double ky = k[my == H ? H : my];
      const double km = std::sqrt(kx2 + ky * ky);
      if (km < cutoff) rt.dmax = my;
      if (d.has_damping && d.mu != 0.0 && km < drag_half) rt.dragmax = my;
      if (d.has_ring && std::fabs(km - d.ring_kf) <= ring_half) {
        if (my < lo) lo = my;
        if (my > hi) hi = my;
      }
    }
    rt.pos_lo = 1; rt.pos_hi = 0; rt.neg_lo = 1; rt.neg_hi = 0;  // empty
    rt.row_start = (int)pl->ring_pos.size();
    if (hi >= lo) {
      const int plo = lo, phi = std::min(hi, H - 1);
      if (phi >= plo) { rt.pos_lo = plo; rt.pos_hi = phi; }
      const int nlo = std::max(N - hi, H), nhi = N - std::max(lo, 1);
      if (nhi >= nlo) { rt.neg_lo = nlo; rt.neg_hi = nhi; }
      for (int iy = rt.pos_lo; iy <= rt.pos_hi; ++iy) pl->ring_pos.push_back(ix * N + iy);
      for (int iy = rt.neg_lo; iy <= rt.neg_hi; ++iy) pl->ring_pos.push_back(ix * N + iy);
    }
  }
  const int n = (int)pl->ring_pos.size();
  pl->ring_mirror.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    const int ix = pl->ring_pos[i] / N, iy = pl->ring_pos[i] % N;
    const int mx = (N - ix) % N, my = (N - iy) % N;
    const RowTab& rt = pl->rows[mx];
    int o = -1;
    if (my >= rt.pos_lo && my <= rt.pos_hi) o = rt.row_start + (my - rt.pos_lo);
    else if (my >= rt.neg_lo && my <= rt.neg_hi)
      o = rt.row_start + (rt.pos_hi >= rt.pos_lo ? rt.pos_hi - rt.pos_lo + 1 : 0) + (my - rt.neg_lo);
    pl->ring_mirror[i] = o;
  }
  const int hpos[4] = {0, H * N, H, H * N + H};
  for (int h = 0; h < 4; ++h) {
    pl->herm_ord[h] = -1;
    for (int i = 0; i < n; ++i)
      if (pl->ring_pos[i] == hpos[h]) pl->herm_ord[h] = i;
  }
  // spectrum bins: numpy linspace(0, k_max, n_bins + 1)
  const double dk = 2 * M_PI / d.L;
  const double kmx = N * dk / 2;
  pl->n_bins = std::min(N / 4, 64);
  pl->edges.assign(pl->n_bins + 1, 0.0);
  const double step = kmx / pl->n_bins;
  for (int i = 0; i <= pl->n_bins; ++i) pl->edges[i] = i * step + 0.0;
  pl->edges[pl->n_bins] = kmx;
  // OU coefficients (ring_forcing.py:112-113)
  if (d.has_ring && d.ring_tau_f > 0) {
    pl->ou_decay = std::exp(-0.0 / d.ring_tau_f);  // set per dt at step time
    pl->ou_vf = 0.0;
  }
}

void layout(sqg_plan* pl) {
  const size_t N = pl->N, H = pl->H, cs = pl->csize;
  const size_t n = std::max<size_t>(pl->ring_pos.size(), 1);
  const size_t full = N * N * cs;
  const size_t half = (H + 1) * N * cs;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o += align256(bytes); return r; };
  pl->off_k1d = take(N * sizeof(double));
  pl->off_k1t = take(N * cs / 2);
  pl->off_tw = take(N * cs);
  pl->off_rows = take(N * sizeof(RowTab));
  pl->off_ring_pos = take(n * sizeof(int));
  pl->off_ring_mirror = take(n * sizeof(int));
  pl->off_ringF = take(4 * n * sizeof(double2));
  pl->off_ring_scale = take(4 * sizeof(double));
  pl->off_ou_state = take(n * sizeof(double2));
  pl->off_ou_init = take(sizeof(int));
  pl->off_status = take(sizeof(unsigned));
  pl->off_step_ctr = take(sizeof(int));
  pl->off_edges = take(65 * sizeof(double));
  pl->off_part = take((size_t)kPartBlocks * 64 * sizeof(double) + 64 * sizeof(double));
  pl->off_acc = take(full);
  pl->off_stage = take(full);
  pl->off_xh = take(4 * half);
  pl->off_jh = take(half);
  pl->off_phys = take(N * N * (cs / 2));
  pl->off_state = take(full);
  pl->off_ctl = take(sizeof(RingCtl));
  const int ns = pl->d.n_scalars;
  pl->n_src_buf = 0;
  for (int s = 0; s < ns; ++s) pl->n_src_buf += pl->d.mean_gradient[s] ? 1 : 0;
  pl->off_uv = take(ns ? full : 0);
  pl->off_xs = take(ns ? 2 * half : 0);
  pl->off_js = take(ns ? half : 0);
  pl->off_sacc = take(ns ? full : 0);
  pl->off_sstage = take(ns ? full : 0);
  pl->off_src = take((size_t)pl->n_src_buf * half);
  pl->off_total = o;
}

KP make_kp(const sqg_plan* pl, double dt) {
  KP kp;
  std::memset(&kp, 0, sizeof(kp));
  const sqg_desc& d = pl->d;
  kp.N = pl->N;
  kp.H = pl->H;
  kp.k1d = wsp<double>(pl, pl->off_k1d);
  kp.k1t = pl->ws + pl->off_k1t;
  kp.tw = pl->ws + pl->off_tw;
  kp.rows = wsp<RowTab>(pl, pl->off_rows);
  kp.inv_n2 = 1.0 / ((double)pl->N * (double)pl->N);
  {
    const double dx = d.L / pl->N;  // the expressions of wavenumbers(): same value bit for bit
    kp.kval = 1.0 / (pl->N * dx);
  }
  kp.alpha = d.alpha;
  kp.akind = pl->akind;
  kp.scheme = d.scheme;
  kp.nu_s = d.nu_p;
  kp.ps = d.p;
  kp.nu_d = d.has_damping ? d.nu_damp : 0.0;
  kp.pd = d.has_damping ? d.p_damp : 8;
  kp.mu = d.has_damping ? d.mu : 0.0;
  kp.dt = dt;
  kp.n_ring = (int)pl->ring_pos.size();
  kp.ring_on = (d.has_ring && kp.n_ring > 0) ? 1 : 0;
  kp.ringF = wsp<double2>(pl, pl->off_ringF);
  kp.status = wsp<unsigned>(pl, pl->off_status);
  return kp;
}

#define SQG_DISPATCH(LOG2N, FN, ...)                  \
  switch (LOG2N) {                                    \
    case 3: return FN<T, 3>(__VA_ARGS__);             \
    case 4: return FN<T, 4>(__VA_ARGS__);             \
    case 5: return FN<T, 5>(__VA_ARGS__);             \
    case 6: return FN<T, 6>(__VA_ARGS__);             \
    case 7: return FN<T, 7>(__VA_ARGS__);             \
    case 8: return FN<T, 8>(__VA_ARGS__);             \
    case 9: return FN<T, 9>(__VA_ARGS__);             \
    case 10: return FN<T, 10>(__VA_ARGS__);           \
    case 11: return FN<T, 11>(__VA_ARGS__);           \
    case 12: return FN<T, 12>(__VA_ARGS__);           \
    default: return cudaErrorInvalidValue;            \
  }

template <typename T>
cudaError_t launch_row_p(int log2n, const KP& kp, const RowArgs& a, cudaStream_t st) {
  SQG_DISPATCH(log2n, launch_row_t, kp, a, st);
}
template <typename T>
cudaError_t launch_col_p(int log2n, const KP& kp, const ColArgs& a, cudaStream_t st, bool ring_only,
                         const CUtensorMap* tm) {
  SQG_DISPATCH(log2n, launch_col_t, kp, a, st, ring_only, tm);
}
template <typename T>
cudaError_t set_attrs_p(int log2n) {
  SQG_DISPATCH(log2n, set_attrs_t);
}
template <typename T>
cudaError_t shape_max_p(int log2n, int* rpc, int* np) {
  SQG_DISPATCH(log2n, shape_max_t, rpc, np);
}

// Timing kinds reported by sqg_timing_read.
enum { TK_ROW_P1 = 0, TK_ROW_STAGE = 1, TK_COL_THETA = 2, TK_ROW_SCALAR = 3, TK_COL_SCALAR = 4, TK_OTHER = 5,
       TK_ROW_LAST = 6, TK_ROW_VEL = 7, TK_COL_VEL = 8, TK_ROW_SCALAR_P1 = 9, TK_COUNT = 10 };

cudaEvent_t next_event(sqg_plan* pl) {
  if (pl->ev_used == pl->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    pl->ev_pool.push_back(e);
  }
  return pl->ev_pool[pl->ev_used++];
}

// With timing on, each launch site issues pl->timing_reps launches of its
// pass back to back (the programmatic dependent launch between them as
// between the passes of a step) inside one pair of events.
template <typename F>
cudaError_t timed(sqg_plan* pl, int kind, cudaStream_t st, F&& f) {
  pl->launches++;
  if (!pl->timing) return f();
  cudaEvent_t a = next_event(pl), b = next_event(pl);
  cudaEventRecord(a, st);
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < pl->timing_reps && e == cudaSuccess; ++r) e = f();
  cudaEventRecord(b, st);
  pl->recs.push_back({kind, a, b, pl->timing_reps});
  return e;
}

int row_kind(const RowArgs& a) {
  if (a.fmode == FM_SCAL) return a.rmode == RM_P1 ? TK_ROW_SCALAR_P1 : TK_ROW_SCALAR;
  if (a.fmode == FM_VEL) return TK_ROW_VEL;
  if (a.fmode != FM_THETA) return TK_OTHER;
  if (a.rmode == RM_P1) return TK_ROW_P1;
  if (a.rmode == RM_STAGE) return a.do_p1 ? TK_ROW_STAGE : TK_ROW_LAST;
  return TK_OTHER;
}

cudaError_t launch_row(sqg_plan* pl, const KP& kp, const RowArgs& a, cudaStream_t st) {
  const int kind = row_kind(a);
  return timed(pl, kind, st, [&] {
    return pl->d.precision == SQG_F64 ? launch_row_p<double>(pl->log2N, kp, a, st)
                                      : launch_row_p<float>(pl->log2N, kp, a, st);
  });
}
cudaError_t launch_col(sqg_plan* pl, const KP& kp, const ColArgs& a, cudaStream_t st, bool ring_only = false) {
  const int kind = a.cmode == CM_THETA ? TK_COL_THETA
                   : (a.cmode == CM_SCAL ? TK_COL_SCALAR : (a.cmode == CM_VEL ? TK_COL_VEL : TK_OTHER));
  // the plan's field stacks xh (theta's four fields, the velocity's two) and
  // xs (a scalar's two gradient fields) have tensor maps
  const CUtensorMap* tm = nullptr;
  if (pl->col_tma && !ring_only && a.cmode != CM_SCALV) {
    if (a.xh == pl->ws + pl->off_xh) tm = &pl->map_xh;
    else if (pl->d.n_scalars > 0 && a.xh == pl->ws + pl->off_xs) tm = &pl->map_xs;
  }
  return timed(pl, kind, st, [&] {
    return pl->d.precision == SQG_F64 ? launch_col_p<double>(pl->log2N, kp, a, st, ring_only, tm)
                                      : launch_col_p<float>(pl->log2N, kp, a, st, ring_only, tm);
  });
}

RowArgs base_row(sqg_plan* pl) {
  RowArgs a;
  std::memset(&a, 0, sizeof(a));
  a.xh = pl->ws + pl->off_xh;
  a.jh = pl->ws + pl->off_jh;
  a.acc = pl->ws + pl->off_acc;
  a.st_in = pl->ws + pl->off_stage;
  a.st_out = pl->ws + pl->off_stage;
  a.fmode = FM_THETA;
  a.rpc = pl->rpc;
  return a;
}

ColArgs base_col(sqg_plan* pl) {
  ColArgs a;
  std::memset(&a, 0, sizeof(a));
  a.cmode = CM_THETA;
  a.xh = pl->ws + pl->off_xh;
  a.jh = pl->ws + pl->off_jh;
  a.np = pl->np;
  return a;
}

// fills the ring-forcing part of the column args for stage s
void ring_args(sqg_plan* pl, ColArgs& a, int s, const void* theta_s, const double* phases, double dt,
               RingCtl* ctl) {
  const sqg_desc& d = pl->d;
  a.ring_cta = 1;
  a.stage = s;
  a.ring_theta = theta_s;
  a.phases = phases;
  a.ring_pos = wsp<int>(pl, pl->off_ring_pos);
  a.ring_mirror = wsp<int>(pl, pl->off_ring_mirror);
  a.ringF = wsp<double2>(pl, pl->off_ringF);
  a.ou_state = wsp<double2>(pl, pl->off_ou_state);
  a.ou_init = wsp<int>(pl, pl->off_ou_init);
  a.ring_amp = d.ring_amplitude;
  a.ring_eps = d.ring_epsilon;
  a.ring_ou = d.ring_tau_f > 0 ? 1 : 0;
  if (a.ring_ou) {
    a.ou_decay = std::exp(-dt / d.ring_tau_f);
    a.ou_vf = std::sqrt(1 - a.ou_decay * a.ou_decay);
  }
  for (int h = 0; h < 4; ++h) a.herm_ord[h] = pl->herm_ord[h];
  a.ring_scale_out = wsp<double>(pl, pl->off_ring_scale);
  a.ctl = ctl;
}

bool ring_active(const sqg_plan* pl) { return pl->d.has_ring && !pl->ring_pos.empty(); }

int check_ready(const sqg_plan* pl) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  if (!pl->ready) return fail(SQG_ERR_WORKSPACE, "workspace not set (call sqg_plan_set_workspace)");
  return SQG_OK;
}

// One RK4 stage: column pass (with ring reduction) then row pass.
int run_stage(sqg_plan* pl, int s, const void* th_n, void* th_out, double dt, const void* extra,
              const double* phases, int stage_write, int do_p1, cudaStream_t st, RingCtl* ctl = nullptr,
              const void* src_phys = nullptr) {
  KP kp = make_kp(pl, dt);
  ColArgs ca = base_col(pl);
  ca.in_real = src_phys;
  if (ring_active(pl)) {
    if (!phases && !ctl) return fail(SQG_ERR_INVALID, "ring forcing needs phases");
    ring_args(pl, ca, s, s == 1 ? th_n : (const void*)(pl->ws + pl->off_stage), phases, dt, ctl);
  }
  SQG_CUDA(launch_col(pl, kp, ca, st));
  RowArgs ra = base_row(pl);
  ra.rmode = RM_STAGE;
  ra.stage = s;
  ra.th_n = th_n;
  ra.th_out = th_out;
  ra.extra = extra;
  ra.stage_write = stage_write;
  ra.do_p1 = do_p1;
  SQG_CUDA(launch_row(pl, kp, ra, st));
  return SQG_OK;
}

int stage_write_mode(const sqg_plan* pl, bool generic) {
  if (generic) return SW_FULL;
  const bool lin = (pl->d.nu_p != 0.0) || (pl->d.has_damping && (pl->d.mu != 0.0 || pl->d.nu_damp != 0.0));
  if (pl->d.scheme == SQG_EXPLICIT_RK4 && lin) return SW_FULL;
  if (ring_active(pl)) return SW_RING;
  return SW_NONE;
}

int run_p1(sqg_plan* pl, const void* th, int fmode, void* xh, cudaStream_t st, double dt = 0.0) {
  KP kp = make_kp(pl, dt);
  RowArgs ra = base_row(pl);
  ra.rmode = RM_P1;
  ra.fmode = fmode;
  ra.th_n = th;
  ra.do_p1 = 1;
  if (xh) ra.xh = xh;
  SQG_CUDA(launch_row(pl, kp, ra, st));
  return SQG_OK;
}

int one_step(sqg_plan* pl, const void* th_in, void* th_out, double dt, const double* phases, bool p1_first,
             cudaStream_t st) {
  int rc;
  if (p1_first) {
    if ((rc = run_p1(pl, th_in, FM_THETA, nullptr, st)) != SQG_OK) return rc;
  }
  const int sw = stage_write_mode(pl, false);
  // stages 1-3 read th_in as theta_n; stage 4 writes th_out (may alias th_in)
  for (int s = 1; s <= 4; ++s) {
    if ((rc = run_stage(pl, s, th_in, th_out, dt, nullptr, phases, sw, s < 4 ? 1 : 0, st)) != SQG_OK) return rc;
  }
  return SQG_OK;
}

}  // namespace

extern "C" {

int sqg_version(void) { return 1; }

const char* sqg_last_error_string(void) { return g_last_error.c_str(); }

int sqg_plan_create(const sqg_desc* desc, sqg_plan** out) {
  if (!desc || !out) return fail(SQG_ERR_INVALID, "null argument");
  const sqg_desc& d = *desc;
  if (d.N % 2 != 0) return fail(SQG_ERR_INVALID, "N must be even, got " + std::to_string(d.N));
  // range first: the power-of-two search below then never shifts past bit 12
  if (d.N < 8 || d.N > 4096 || (d.N & (d.N - 1)) != 0)
    return fail(SQG_ERR_INVALID, "N must be a power of two in [8, 4096], got " + std::to_string(d.N));
  int log2n = 0;
  while ((1 << log2n) < d.N) ++log2n;
  if (!(d.alpha >= -2 && d.alpha <= 2)) return fail(SQG_ERR_INVALID, "alpha must be in [-2, 2], got " + std::to_string(d.alpha));
  if (d.p != 2 && d.p != 4 && d.p != 8) return fail(SQG_ERR_INVALID, "p must be 2, 4, or 8, got " + std::to_string(d.p));
  if (d.has_damping && d.p_damp != 2 && d.p_damp != 4 && d.p_damp != 8)
    return fail(SQG_ERR_INVALID, "p must be 2, 4, or 8, got " + std::to_string(d.p_damp));
  if (d.precision != SQG_F64 && d.precision != SQG_F32) return fail(SQG_ERR_INVALID, "bad precision");
  if (d.scheme != SQG_EXPLICIT_RK4 && d.scheme != SQG_IF_RK4) return fail(SQG_ERR_INVALID, "bad scheme");
  if (!(d.L > 0)) return fail(SQG_ERR_INVALID, "L must be positive");
  if (d.n_scalars < 0 || d.n_scalars > SQG_MAX_SCALARS) return fail(SQG_ERR_INVALID, "n_scalars out of range");
  sqg_plan* pl = new sqg_plan();
  pl->d = d;
  pl->N = d.N;
  pl->H = d.N / 2;
  pl->log2N = log2n;
  pl->csize = d.precision == SQG_F64 ? 16 : 8;
  pl->akind = alpha_kind(d.alpha);
  build_tables(pl);
  layout(pl);
  *out = pl;
  return SQG_OK;
}

int sqg_plan_destroy(sqg_plan* pl) {
  if (!pl) return SQG_OK;
  if (pl->graph_exec) cudaGraphExecDestroy(pl->graph_exec);
  for (cudaEvent_t e : pl->ev_pool) cudaEventDestroy(e);
  if (pl->cap_stream) cudaStreamDestroy(pl->cap_stream);
  if (pl->ev_in) cudaEventDestroy(pl->ev_in);
  if (pl->ev_out) cudaEventDestroy(pl->ev_out);
  delete pl;
  return SQG_OK;
}

int sqg_plan_workspace_bytes(const sqg_plan* pl, size_t* bytes) {
  if (!pl || !bytes) return fail(SQG_ERR_INVALID, "null argument");
  *bytes = pl->off_total;
  return SQG_OK;
}

int sqg_plan_buffer(const sqg_plan* pl, int32_t which, size_t* offset, size_t* bytes) {
  if (!pl || !offset || !bytes) return fail(SQG_ERR_INVALID, "null argument");
  const size_t full = (size_t)pl->N * pl->N * pl->csize;
  switch (which) {
    case SQG_BUF_STAGE: *offset = pl->off_stage; *bytes = full; break;
    case SQG_BUF_UV: *offset = pl->off_uv; *bytes = pl->d.n_scalars ? full : 0; break;
    case SQG_BUF_RING_FORCE: *offset = pl->off_ringF; *bytes = pl->ring_pos.size() * sizeof(double2); break;
    case SQG_BUF_STATUS: *offset = pl->off_status; *bytes = sizeof(unsigned); break;
    default: return fail(SQG_ERR_INVALID, "unknown buffer");
  }
  return SQG_OK;
}

// ---- tensor maps of the column passes' field stacks ----
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// nf fields of (N/2+1) x N complex from base, as 32-bit elements; a box is a
// column pair (2 complex) over min(N/2, 256) rows.
bool encode_field_stack(CUtensorMap* m, void* base, int N, size_t cs, int nf, CUtensorMapL2promotion promo) {
  EncodeTiledFn f = encode_tiled();
  if (!f || ((uintptr_t)base & 15)) return false;
  const int H = N / 2;
  const cuuint64_t dims[3] = {(cuuint64_t)N * cs / 4, (cuuint64_t)H + 1, (cuuint64_t)nf};
  const cuuint64_t strides[2] = {(cuuint64_t)N * cs, (cuuint64_t)(H + 1) * N * cs};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * cs / 4), (cuuint32_t)(H < 256 ? H : 256), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Column passes at N >= kColTmaMinN take their half columns as TMA tiles
// when both maps encode; SQG_COL_TMA=0 in the environment keeps the cp.async
// gathers.  Measured at N = 4096 (FP32, per launch): theta column pass 208 ->
// 183 us, scalar column pass 136.5 -> 121 us, velocity column pass 96 ->
// 80 us; FP64 theta 488 -> 461 us.  The tiles' L2 promotion (none, 128 or
// 256 bytes) made no measurable difference.
void bind_col_maps(sqg_plan* pl) {
  pl->col_tma = false;
  if (pl->N < kColTmaMinN || pl->ws_bytes < pl->off_total) return;
  const char* env = std::getenv("SQG_COL_TMA");
  if (env && std::string(env) == "0") return;
  const CUtensorMapL2promotion promo = CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
  std::memset(&pl->map_xh, 0, sizeof(CUtensorMap));
  std::memset(&pl->map_xs, 0, sizeof(CUtensorMap));
  bool ok = encode_field_stack(&pl->map_xh, pl->ws + pl->off_xh, pl->N, pl->csize, 4, promo);
  if (ok && pl->d.n_scalars > 0) ok = encode_field_stack(&pl->map_xs, pl->ws + pl->off_xs, pl->N, pl->csize, 2, promo);
  pl->col_tma = ok;
}

int sqg_plan_set_workspace(sqg_plan* pl, void* ws, size_t bytes, void* stream) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  if (!ws) return fail(SQG_ERR_WORKSPACE, "null workspace");
  if (bytes < pl->off_total) return fail(SQG_ERR_WORKSPACE, "workspace too small");
  if (((uintptr_t)ws) & 255) return fail(SQG_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  pl->ws = (unsigned char*)ws;
  pl->ws_bytes = bytes;
  const int N = pl->N;
  // host staging of the tables
  std::vector<unsigned char> host(pl->off_acc, 0);
  std::memcpy(host.data() + pl->off_k1d, pl->k1d.data(), N * sizeof(double));
  if (pl->d.precision == SQG_F64) {
    std::memcpy(host.data() + pl->off_k1t, pl->k1d.data(), N * sizeof(double));
    std::vector<double2> tw(N);
    for (int k = 0; k < N; ++k) {
      const long double ang = 2.0L * 3.14159265358979323846264338327950288L * k / N;
      tw[k] = make_double2((double)cosl(ang), (double)-sinl(ang));
    }
    std::memcpy(host.data() + pl->off_tw, tw.data(), N * sizeof(double2));
  } else {
    std::vector<float> kf(N);
    for (int i = 0; i < N; ++i) kf[i] = (float)pl->k1d[i];
    std::memcpy(host.data() + pl->off_k1t, kf.data(), N * sizeof(float));
    std::vector<float2> tw(N);
    for (int k = 0; k < N; ++k) {
      const long double ang = 2.0L * 3.14159265358979323846264338327950288L * k / N;
      tw[k] = make_float2((float)cosl(ang), (float)-sinl(ang));
    }
    std::memcpy(host.data() + pl->off_tw, tw.data(), N * sizeof(float2));
  }
  std::memcpy(host.data() + pl->off_rows, pl->rows.data(), N * sizeof(RowTab));
  if (!pl->ring_pos.empty()) {
    std::memcpy(host.data() + pl->off_ring_pos, pl->ring_pos.data(), pl->ring_pos.size() * sizeof(int));
    std::memcpy(host.data() + pl->off_ring_mirror, pl->ring_mirror.data(), pl->ring_mirror.size() * sizeof(int));
  }
  std::memcpy(host.data() + pl->off_edges, pl->edges.data(), pl->edges.size() * sizeof(double));
  SQG_CUDA(cudaMemcpyAsync(ws, host.data(), pl->off_acc, cudaMemcpyHostToDevice, st));
  SQG_CUDA(cudaStreamSynchronize(st));
  if (pl->d.precision == SQG_F64) { SQG_CUDA(set_attrs_p<double>(pl->log2N)); }
  else { SQG_CUDA(set_attrs_p<float>(pl->log2N)); }
  bind_col_maps(pl);
  if (pl->graph_exec) {
    cudaGraphExecDestroy(pl->graph_exec);
    pl->graph_exec = nullptr;
  }
  pl->ready = true;  // (graph captures reference workspace addresses)
  return SQG_OK;
}

int sqg_ring_mode_count(const sqg_plan* pl, int32_t* n) {
  if (!pl || !n) return fail(SQG_ERR_INVALID, "null argument");
  *n = pl->d.has_ring ? (int32_t)pl->ring_pos.size() : 0;
  return SQG_OK;
}

int sqg_ring_modes(const sqg_plan* pl, int32_t* ix, int32_t* iy) {
  if (!pl || !ix || !iy) return fail(SQG_ERR_INVALID, "null argument");
  for (size_t i = 0; i < pl->ring_pos.size(); ++i) {
    ix[i] = pl->ring_pos[i] / pl->N;
    iy[i] = pl->ring_pos[i] % pl->N;
  }
  return SQG_OK;
}

// Host copies of the grid tables (CPU-side checks of the masks).
int sqg_plan_host_tables(const sqg_plan* pl, double* k1d, int32_t* dmax, int32_t* dragmax) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  for (int i = 0; i < pl->N; ++i) {
    if (k1d) k1d[i] = pl->k1d[i];
    if (dmax) dmax[i] = pl->rows[i].dmax;
    if (dragmax) dragmax[i] = pl->rows[i].dragmax;
  }
  return SQG_OK;
}

int sqg_plan_shape(const sqg_plan* pl, int32_t* rpc, int32_t* np, int32_t* max_rpc, int32_t* max_np) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  int mr = 0, mn = 0;
  if (pl->d.precision == SQG_F64) shape_max_p<double>(pl->log2N, &mr, &mn);
  else shape_max_p<float>(pl->log2N, &mr, &mn);
  if (rpc) *rpc = pl->rpc > 0 ? pl->rpc : mr;
  if (np) *np = pl->np > 0 ? pl->np : mn;
  if (max_rpc) *max_rpc = mr;
  if (max_np) *max_np = mn;
  return SQG_OK;
}

int sqg_plan_set_shape(sqg_plan* pl, int32_t rpc, int32_t np) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  int mr = 0, mn = 0;
  if (pl->d.precision == SQG_F64) shape_max_p<double>(pl->log2N, &mr, &mn);
  else shape_max_p<float>(pl->log2N, &mr, &mn);
  auto ok = [](int v, int m) { return v == 0 || (v >= 1 && v <= m && (m % v) == 0 && (v & (v - 1)) == 0); };
  if (!ok(rpc, mr)) return fail(SQG_ERR_INVALID, "rpc must be 0 or a power-of-two divisor of " + std::to_string(mr));
  if (!ok(np, mn)) return fail(SQG_ERR_INVALID, "np must be 0 or a power-of-two divisor of " + std::to_string(mn));
  if (pl->rpc != rpc || pl->np != np) {
    pl->rpc = rpc;
    pl->np = np;
    if (pl->graph_exec) {  // the captured step holds the old launch shapes
      cudaGraphExecDestroy(pl->graph_exec);
      pl->graph_exec = nullptr;
    }
  }
  return SQG_OK;
}

// Times the transform passes of one right-hand side (row inverse pass,
// column pass, row pass) for every launch shape on the plan's own buffers and
// keeps the fastest.  Blocks the calling thread (events are synchronised).
int sqg_plan_autotune(sqg_plan* pl, int32_t reps, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (reps < 1) reps = 1;
  cudaStream_t st = (cudaStream_t)stream;
  int mr = 0, mn = 0;
  if (pl->d.precision == SQG_F64) shape_max_p<double>(pl->log2N, &mr, &mn);
  else shape_max_p<float>(pl->log2N, &mr, &mn);
  void* th = pl->ws + pl->off_state;  // scratch input (zeroed) and output inside the workspace
  void* out = pl->ws + pl->off_stage;
  const size_t full = (size_t)pl->N * pl->N * pl->csize;
  SQG_CUDA(cudaMemsetAsync(th, 0, full, st));
  const bool timing = pl->timing;
  pl->timing = false;
  const int r0 = pl->rpc, n0 = pl->np;
  auto one = [&]() -> int {
    int e = run_p1(pl, th, FM_THETA, nullptr, st);
    if (e) return e;
    KP kp = make_kp(pl, 0.0);
    kp.ring_on = 0;
    ColArgs ca = base_col(pl);
    SQG_CUDA(launch_col(pl, kp, ca, st));
    RowArgs ra = base_row(pl);
    ra.rmode = RM_RHS;
    ra.stage = 1;
    ra.th_n = th;
    ra.rhs_out = out;
    ra.do_p1 = 0;
    SQG_CUDA(launch_row(pl, kp, ra, st));
    return SQG_OK;
  };
  cudaEvent_t e0, e1;
  SQG_CUDA(cudaEventCreate(&e0));
  SQG_CUDA(cudaEventCreate(&e1));
  // every shape is timed in three interleaved rounds and keeps its fastest
  // round, so that a clock ramp or a stray slow round early on does not
  // decide the choice
  std::vector<std::pair<int, int>> shapes;
  for (int r = mr; r >= 1; r /= 2)
    for (int n = mn; n >= 1; n /= 2) shapes.push_back({r, n});
  std::vector<float> t_best(shapes.size(), 1e30f);
  for (int round = 0; round < 3 && rc == SQG_OK; ++round) {
    for (size_t i = 0; i < shapes.size() && rc == SQG_OK; ++i) {
      pl->rpc = shapes[i].first;
      pl->np = shapes[i].second;
      if ((rc = one()) != SQG_OK) break;  // warm-up
      cudaEventRecord(e0, st);
      for (int k = 0; k < reps && rc == SQG_OK; ++k) rc = one();
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(SQG_ERR_CUDA, "autotune: event"); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < t_best[i]) t_best[i] = ms;
    }
  }
  float best = 1e30f;
  int br = mr, bn = mn;
  for (size_t i = 0; i < shapes.size(); ++i)
    if (t_best[i] < best) { best = t_best[i]; br = shapes[i].first; bn = shapes[i].second; }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pl->timing = timing;
  pl->rpc = r0;
  pl->np = n0;
  if (rc != SQG_OK) return rc;
  return sqg_plan_set_shape(pl, br == mr ? 0 : br, bn == mn ? 0 : bn);
}

int sqg_rhs(sqg_plan* pl, const void* theta, void* rhs, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !rhs) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  pl->launches = 0;
  if ((rc = run_p1(pl, theta, FM_THETA, nullptr, st)) != SQG_OK) return rc;
  KP kp = make_kp(pl, 0.0);
  kp.ring_on = 0;
  ColArgs ca = base_col(pl);
  SQG_CUDA(launch_col(pl, kp, ca, st));
  RowArgs ra = base_row(pl);
  ra.rmode = RM_RHS;
  ra.stage = 1;
  ra.th_n = theta;
  ra.rhs_out = rhs;
  ra.do_p1 = 0;
  SQG_CUDA(launch_row(pl, kp, ra, st));
  return SQG_OK;
}

int sqg_step(sqg_plan* pl, const void* th_in, void* th_out, double dt, const double* phases, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!th_in || !th_out) return fail(SQG_ERR_INVALID, "null pointer");
  pl->launches = 0;
  return one_step(pl, th_in, th_out, dt, phases, true, (cudaStream_t)stream);
}

int sqg_stage_begin(sqg_plan* pl, const void* th_in, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  pl->launches = 0;
  rc = run_p1(pl, th_in, FM_THETA, nullptr, (cudaStream_t)stream);
  if (rc == SQG_OK) pl->stage_begun = true;
  return rc;
}

int sqg_stage(sqg_plan* pl, int32_t s, const void* th_in, void* th_out, double dt, const void* extra,
              const double* phases, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!pl->stage_begun) return fail(SQG_ERR_STATE, "sqg_stage before sqg_stage_begin");
  if (s < 1 || s > 4) return fail(SQG_ERR_INVALID, "stage must be 1..4");
  rc = run_stage(pl, s, th_in, th_out, dt, extra, phases, stage_write_mode(pl, true), s < 4 ? 1 : 0,
                 (cudaStream_t)stream);
  if (s == 4) pl->stage_begun = false;
  return rc;
}

int sqg_stage_physical(sqg_plan* pl, int32_t s, const void* th_in, void* th_out, double dt, const void* src,
                       const double* phases, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!pl->stage_begun) return fail(SQG_ERR_STATE, "sqg_stage_physical before sqg_stage_begin");
  if (s < 1 || s > 4) return fail(SQG_ERR_INVALID, "stage must be 1..4");
  if (!src) return fail(SQG_ERR_INVALID, "null source field");
  rc = run_stage(pl, s, th_in, th_out, dt, nullptr, phases, stage_write_mode(pl, true), s < 4 ? 1 : 0,
                 (cudaStream_t)stream, nullptr, src);
  if (s == 4) pl->stage_begun = false;
  return rc;
}

int sqg_multistep(sqg_plan* pl, void* theta, int32_t n_steps, double dt, const double* phases, int32_t use_graph,
                  void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta) return fail(SQG_ERR_INVALID, "null pointer");
  if (n_steps < 0) return fail(SQG_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return SQG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int n_ring = (int)pl->ring_pos.size();
  const bool ring = ring_active(pl);
  if (ring && !phases) return fail(SQG_ERR_INVALID, "ring forcing needs phases");
  pl->launches = 0;
  const int sw = stage_write_mode(pl, false);
  if (!use_graph || pl->timing) {
    if ((rc = run_p1(pl, theta, FM_THETA, nullptr, st)) != SQG_OK) return rc;
    for (int n = 0; n < n_steps; ++n) {
      const double* ph = ring ? phases + (size_t)n * n_ring : nullptr;
      for (int s = 1; s <= 4; ++s) {
        const int do_p1 = (s < 4 || n + 1 < n_steps) ? 1 : 0;
        if ((rc = run_stage(pl, s, theta, theta, dt, nullptr, ph, sw, do_p1, st)) != SQG_OK) return rc;
      }
    }
    return SQG_OK;
  }
  // CUDA graph of one steady-state step, captured on the plan's own stream
  // over the plan's state buffer (stage 4 also prepares the next step; the
  // ring phases of step n are read through the device control block).
  void* state = pl->ws + pl->off_state;
  RingCtl* ctl = wsp<RingCtl>(pl, pl->off_ctl);
  const size_t full = (size_t)pl->N * pl->N * pl->csize;
  if (!pl->cap_stream) {
    SQG_CUDA(cudaStreamCreateWithFlags(&pl->cap_stream, cudaStreamNonBlocking));
    SQG_CUDA(cudaEventCreateWithFlags(&pl->ev_in, cudaEventDisableTiming));
    SQG_CUDA(cudaEventCreateWithFlags(&pl->ev_out, cudaEventDisableTiming));
  }
  cudaStream_t cs = pl->cap_stream;
  if (!pl->graph_exec || pl->graph_dt != dt) {
    if (pl->graph_exec) {
      cudaGraphExecDestroy(pl->graph_exec);
      pl->graph_exec = nullptr;
    }
    cudaGraph_t g;
    SQG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int64_t saved = pl->launches;
    for (int s = 1; s <= 4 && rc == SQG_OK; ++s)
      rc = run_stage(pl, s, state, state, dt, nullptr, nullptr, sw, 1, cs, ring ? ctl : nullptr);
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    pl->launches = saved;
    if (rc != SQG_OK) return rc;
    if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&pl->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
    pl->graph_dt = dt;
  }
  SQG_CUDA(cudaMemcpyAsync(state, theta, full, cudaMemcpyDeviceToDevice, st));
  if (ring) {
    k_set_ctl<<<1, 1, 0, st>>>(ctl, phases);
    SQG_CUDA(cudaGetLastError());
  }
  if ((rc = run_p1(pl, state, FM_THETA, nullptr, st)) != SQG_OK) return rc;
  SQG_CUDA(cudaEventRecord(pl->ev_in, st));
  SQG_CUDA(cudaStreamWaitEvent(cs, pl->ev_in, 0));
  for (int n = 0; n < n_steps; ++n) {
    SQG_CUDA(cudaGraphLaunch(pl->graph_exec, cs));
    pl->launches += 8;
  }
  SQG_CUDA(cudaEventRecord(pl->ev_out, cs));
  SQG_CUDA(cudaStreamWaitEvent(st, pl->ev_out, 0));
  SQG_CUDA(cudaMemcpyAsync(theta, state, full, cudaMemcpyDeviceToDevice, st));
  return SQG_OK;
}

int sqg_velocity(sqg_plan* pl, const void* theta, void* u, void* v, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !u || !v) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = run_p1(pl, theta, FM_VEL, nullptr, st)) != SQG_OK) return rc;
  KP kp = make_kp(pl, 0.0);
  ColArgs ca = base_col(pl);
  ca.cmode = CM_VEL;
  ca.out0 = u;
  ca.out1 = v;
  SQG_CUDA(launch_col(pl, kp, ca, st));
  return SQG_OK;
}

int sqg_to_physical(sqg_plan* pl, const void* field_hat, void* field, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!field_hat || !field) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = run_p1(pl, field_hat, FM_PHYS1, nullptr, st)) != SQG_OK) return rc;
  KP kp = make_kp(pl, 0.0);
  ColArgs ca = base_col(pl);
  ca.cmode = CM_PHYS1;
  ca.out0 = field;
  SQG_CUDA(launch_col(pl, kp, ca, st));
  return SQG_OK;
}

static int linear_term(sqg_plan* pl, const void* theta, void* out, double nu, int pw, double mu, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !out) return fail(SQG_ERR_INVALID, "null pointer");
  KP kp = make_kp(pl, 0.0);
  cudaStream_t st = (cudaStream_t)stream;
  if (pl->d.precision == SQG_F64)
    k_linear<double><<<4 * kPartBlocks, 256, 0, st>>>(kp, nu, pw, mu, (const double2*)theta, (double2*)out);
  else
    k_linear<float><<<4 * kPartBlocks, 256, 0, st>>>(kp, nu, pw, mu, (const float2*)theta, (float2*)out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_damping(sqg_plan* pl, const void* theta, void* out, void* stream) {
  if (pl && !pl->d.has_damping) return fail(SQG_ERR_INVALID, "plan carries no damping");
  return linear_term(pl, theta, out, pl ? pl->d.nu_damp : 0.0, pl ? pl->d.p_damp : 8, pl ? pl->d.mu : 0.0, stream);
}

int sqg_hyperviscosity(sqg_plan* pl, const void* theta, void* out, void* stream) {
  return linear_term(pl, theta, out, pl ? pl->d.nu_p : 0.0, pl ? pl->d.p : 8, 0.0, stream);
}

int sqg_to_spectral(sqg_plan* pl, const void* field, void* field_hat, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!field || !field_hat) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  KP kp = make_kp(pl, 0.0);
  ColArgs ca = base_col(pl);
  ca.cmode = CM_FWD;
  ca.in_real = field;
  SQG_CUDA(launch_col(pl, kp, ca, st));
  RowArgs ra = base_row(pl);
  ra.rmode = RM_SPEC;
  ra.rhs_out = field_hat;
  SQG_CUDA(launch_row(pl, kp, ra, st));
  return SQG_OK;
}

int sqg_inner(sqg_plan* pl, const void* a, const void* b, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!a || !b || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = wsp<double>(pl, pl->off_part);
  if (pl->d.precision == SQG_F64)
    k_inner_partial<double><<<kPartBlocks, 256, 0, st>>>(pl->N, (const double2*)a, (const double2*)b, part);
  else
    k_inner_partial<float><<<kPartBlocks, 256, 0, st>>>(pl->N, (const float2*)a, (const float2*)b, part);
  k_var_final<<<1, 256, 0, st>>>(kPartBlocks, pl->N, part, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_ring_forcing(sqg_plan* pl, const void* theta, const double* phases, double dt, void* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t full = (size_t)pl->N * pl->N * pl->csize;
  SQG_CUDA(cudaMemsetAsync(out, 0, full, st));
  if (!ring_active(pl)) return SQG_OK;
  if (!phases) return fail(SQG_ERR_INVALID, "ring forcing needs phases");
  KP kp = make_kp(pl, dt);
  ColArgs ca = base_col(pl);
  ring_args(pl, ca, 1, theta, phases, dt, nullptr);
  SQG_CUDA(launch_col(pl, kp, ca, st, true));
  const int n = (int)pl->ring_pos.size();
  if (pl->d.precision == SQG_F64)
    k_ring_scatter<double><<<(n + 255) / 256, 256, 0, st>>>(n, wsp<int>(pl, pl->off_ring_pos), kp.ringF, (double2*)out);
  else
    k_ring_scatter<float><<<(n + 255) / 256, 256, 0, st>>>(n, wsp<int>(pl, pl->off_ring_pos), kp.ringF, (float2*)out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_ring_substeps(sqg_plan* pl, void* theta, int32_t n_sub, double dt_sub, const double* phases, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta) return fail(SQG_ERR_INVALID, "null pointer");
  if (!ring_active(pl)) return fail(SQG_ERR_INVALID, "the plan carries no ring forcing");
  if (pl->d.ring_tau_f > 0.0) return fail(SQG_ERR_INVALID, "forcing sub-steps need tau_f = 0 (white-in-time forcing)");
  if (n_sub < 0) return fail(SQG_ERR_INVALID, "n_sub must be >= 0");
  if (n_sub == 0) return SQG_OK;
  if (!phases) return fail(SQG_ERR_INVALID, "forcing sub-steps need phases");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = (int)pl->ring_pos.size();
  const int4 ho = make_int4(pl->herm_ord[0], pl->herm_ord[1], pl->herm_ord[2], pl->herm_ord[3]);
  double2* F = wsp<double2>(pl, pl->off_ringF);  // scratch: first n entries of the stage forcing table
  const int* pos = wsp<int>(pl, pl->off_ring_pos);
  const int* mir = wsp<int>(pl, pl->off_ring_mirror);
  if (pl->d.precision == SQG_F64)
    SQG_CUDA(launch_pdl(k_ring_substeps<double>, dim3(1), dim3(256), 0, st, pl->N, n, pos, mir, ho,
                        pl->d.ring_amplitude, pl->d.ring_epsilon, n_sub, dt_sub, phases, (double2*)theta, F));
  else
    SQG_CUDA(launch_pdl(k_ring_substeps<float>, dim3(1), dim3(256), 0, st, pl->N, n, pos, mir, ho,
                        pl->d.ring_amplitude, pl->d.ring_epsilon, n_sub, dt_sub, phases, (float2*)theta, F));
  pl->launches++;
  return SQG_OK;
}

int sqg_max_speed(sqg_plan* pl, const void* u, const void* v, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!u || !v || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = wsp<double>(pl, pl->off_part);
  const size_t nn = (size_t)pl->N * pl->N;
  if (pl->d.precision == SQG_F64)
    k_speedmax_partial<double><<<kPartBlocks, 256, 0, st>>>((const double*)u, (const double*)v, nn, part);
  else
    k_speedmax_partial<float><<<kPartBlocks, 256, 0, st>>>((const float*)u, (const float*)v, nn, part);
  k_nanmax_final<<<1, 256, 0, st>>>(kPartBlocks, part, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_spectrum_absmax(sqg_plan* pl, const void* theta, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = wsp<double>(pl, pl->off_part);
  const size_t nn = (size_t)pl->N * pl->N;
  if (pl->d.precision == SQG_F64)
    k_cabsmax_partial<double2><<<kPartBlocks, 256, 0, st>>>((const double2*)theta, nn, part);
  else
    k_cabsmax_partial<float2><<<kPartBlocks, 256, 0, st>>>((const float2*)theta, nn, part);
  k_nanmax_final<<<1, 256, 0, st>>>(kPartBlocks, part, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_diagnostics(sqg_plan* pl, const void* theta, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  KP kp = make_kp(pl, 0.0);
  double* part = wsp<double>(pl, pl->off_part);
  double* maxv = part + (size_t)kPartBlocks * 64;
  // max |theta| in physical space
  void* phys = pl->ws + pl->off_phys;
  if ((rc = sqg_to_physical(pl, theta, phys, stream)) != SQG_OK) return rc;
  const size_t nn = (size_t)pl->N * pl->N;
  if (pl->d.precision == SQG_F64)
    k_absmax_partial<double><<<kPartBlocks, 256, 0, st>>>((const double*)phys, nn, part);
  else
    k_absmax_partial<float><<<kPartBlocks, 256, 0, st>>>((const float*)phys, nn, part);
  k_absmax_final<<<1, 256, 0, st>>>(kPartBlocks, part, maxv);
  if (pl->d.precision == SQG_F64)
    k_diag_partial<double><<<kPartBlocks, 256, 0, st>>>(kp, (const double2*)theta, part);
  else
    k_diag_partial<float><<<kPartBlocks, 256, 0, st>>>(kp, (const float2*)theta, part);
  k_diag_final<<<1, 256, 0, st>>>(kPartBlocks, pl->N, part, maxv, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_energy_spectrum(sqg_plan* pl, const void* theta, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!theta || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  KP kp = make_kp(pl, 0.0);
  double* part = wsp<double>(pl, pl->off_part);
  const double* edges = wsp<double>(pl, pl->off_edges);
  if (pl->d.precision == SQG_F64)
    k_spectrum_partial<double><<<kPartBlocks, 256, 0, st>>>(kp, (const double2*)theta, edges, pl->n_bins, part);
  else
    k_spectrum_partial<float><<<kPartBlocks, 256, 0, st>>>(kp, (const float2*)theta, edges, pl->n_bins, part);
  k_spectrum_final<<<1, 64, 0, st>>>(kPartBlocks, pl->n_bins, part, edges, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_scalar_variance(sqg_plan* pl, const void* s_hat, double* out, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!s_hat || !out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = wsp<double>(pl, pl->off_part);
  if (pl->d.precision == SQG_F64)
    k_var_partial<double><<<kPartBlocks, 256, 0, st>>>(pl->N, (const double2*)s_hat, part);
  else
    k_var_partial<float><<<kPartBlocks, 256, 0, st>>>(pl->N, (const float2*)s_hat, part);
  k_var_final<<<1, 256, 0, st>>>(kPartBlocks, pl->N, part, out);
  SQG_CUDA(cudaGetLastError());
  return SQG_OK;
}

int sqg_scalars_step(sqg_plan* pl, const void* theta_new, const void* const* s_in, void* const* s_out, double dt,
                     void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  const int ns = pl->d.n_scalars;
  if (ns == 0) return SQG_OK;
  if (!theta_new || !s_in || !s_out) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  KP kp = make_kp(pl, dt);
  kp.ring_on = 0;
  void* uv = pl->ws + pl->off_uv;
  void* xs = pl->ws + pl->off_xs;
  void* js = pl->ws + pl->off_js;
  // 1. velocity of theta_new (frozen over the scalar stages) and the
  //    mean-gradient source spectra
  {
    RowArgs ra = base_row(pl);
    ra.rmode = RM_P1;
    ra.fmode = FM_VEL;
    ra.th_n = theta_new;
    ra.do_p1 = 1;
    int k = 0;
    for (int s = 0; s < ns; ++s) {
      if (!pl->d.mean_gradient[s]) continue;
      ra.src_out[k] = pl->ws + pl->off_src + (size_t)k * (pl->H + 1) * pl->N * pl->csize;
      ra.gx[k] = pl->d.grad_x[s];
      ra.gy[k] = pl->d.grad_y[s];
      ++k;
    }
    ra.n_src = k;
    SQG_CUDA(launch_row(pl, kp, ra, st));
    ColArgs ca = base_col(pl);
    ca.cmode = CM_VEL;
    ca.out0 = uv;
    ca.out1 = nullptr;
    SQG_CUDA(launch_col(pl, kp, ca, st));
  }
  // 2. RK4 of each scalar
  int ksrc = 0;
  for (int s = 0; s < ns; ++s) {
    const void* src = nullptr;
    if (pl->d.mean_gradient[s]) {
      src = pl->ws + pl->off_src + (size_t)ksrc * (pl->H + 1) * pl->N * pl->csize;
      ++ksrc;
    }
    RowArgs p1 = base_row(pl);
    p1.rmode = RM_P1;
    p1.fmode = FM_SCAL;
    p1.th_n = s_in[s];
    p1.do_p1 = 1;
    p1.xh = xs;
    SQG_CUDA(launch_row(pl, kp, p1, st));
    const bool explicit_lin = pl->d.scheme == SQG_EXPLICIT_RK4 && pl->d.kappa[s] != 0.0;
    for (int stg = 1; stg <= 4; ++stg) {
      ColArgs ca = base_col(pl);
      ca.cmode = CM_SCAL;
      ca.xh = xs;
      ca.jh = js;
      ca.uv = uv;
      SQG_CUDA(launch_col(pl, kp, ca, st));
      RowArgs ra = base_row(pl);
      ra.rmode = RM_STAGE;
      ra.fmode = FM_SCAL;
      ra.stage = stg;
      ra.th_n = s_in[s];
      ra.th_out = s_out[s];
      ra.acc = pl->ws + pl->off_sacc;
      ra.st_in = pl->ws + pl->off_sstage;
      ra.st_out = pl->ws + pl->off_sstage;
      ra.jh = js;
      ra.xh = xs;
      ra.kappa = pl->d.kappa[s];
      ra.src_h = src;
      ra.stage_write = explicit_lin ? SW_FULL : SW_NONE;
      ra.do_p1 = stg < 4 ? 1 : 0;
      KP kps = kp;
      kps.ring_on = 0;
      SQG_CUDA(launch_row(pl, kps, ra, st));
    }
  }
  return SQG_OK;
}

int sqg_check_status(sqg_plan* pl, uint32_t* flags, void* stream) {
  int rc = check_ready(pl);
  if (rc) return rc;
  if (!flags) return fail(SQG_ERR_INVALID, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned h = 0;
  SQG_CUDA(cudaMemcpyAsync(&h, pl->ws + pl->off_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SQG_CUDA(cudaStreamSynchronize(st));
  SQG_CUDA(cudaMemsetAsync(pl->ws + pl->off_status, 0, sizeof(unsigned), st));
  *flags = h;
  return SQG_OK;
}

int sqg_set_timing(sqg_plan* pl, int32_t enable) {
  if (!pl) return fail(SQG_ERR_INVALID, "null plan");
  if (enable < 0) return fail(SQG_ERR_INVALID, "enable must be >= 0");
  if (enable > 1 && pl->d.has_ring && pl->d.ring_tau_f > 0)
    return fail(SQG_ERR_INVALID, "repeated timing launches would advance the forcing's OU state");
  pl->timing = enable != 0;
  pl->timing_reps = enable > 1 ? enable : 1;
  pl->recs.clear();
  pl->ev_used = 0;
  return SQG_OK;
}

int sqg_timing_read(sqg_plan* pl, double* ms, int64_t* count, int32_t nkinds) {
  if (!pl || !ms || !count) return fail(SQG_ERR_INVALID, "null argument");
  for (int k = 0; k < nkinds; ++k) { ms[k] = 0.0; count[k] = 0; }
  for (const auto& r : pl->recs) {
    SQG_CUDA(cudaEventSynchronize(r.b));
    float t = 0.f;
    SQG_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kind < nkinds) { ms[r.kind] += t; count[r.kind] += r.reps; }
  }
  pl->recs.clear();
  pl->ev_used = 0;
  return SQG_OK;
}

int sqg_last_launch_count(const sqg_plan* pl, int64_t* n) {
  if (!pl || !n) return fail(SQG_ERR_INVALID, "null argument");
  *n = pl->launches;
  return SQG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sqg_rhs_noalloc: the core RHS for callers that cannot allocate device memory.
//
// Some host programs must not call cudaMalloc from the code that calls this
// library -- e.g. a coupler or plugin host that reserves all device memory up
// front through its own allocator, or a latency-critical loop where
// cudaMalloc/cudaFree are banned because they can synchronise the device.
// Such a caller passes only its input and output spectra.  Everything else
// (grid tables and the intermediate transformed fields) lives in the
// file-scope array below, which every GPU that loads this library holds for
// the life of the process.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SQG_NOALLOC_SCRATCH_BYTES];

// Grid tables of the no-allocation path, computed on the device with the
// same float64 expressions the host path uses (round-to-nearest intrinsics
// keep the compiler from contracting them into FMAs, so the dealiasing mask
// edges are the reference's bit for bit).
template <typename T>
__global__ void k_noalloc_tables(int N, double L, double* k1d, T* k1t, typename Cplx<T>::type* tw, RowTab* rows,
                                 unsigned* status) {
  using C = typename Cplx<T>::type;
  const int H = N / 2;
  const double dx = __ddiv_rn(L, (double)N);
  const double val = __ddiv_rn(1.0, __dmul_rn((double)N, dx));
  const int npos = (N - 1) / 2 + 1;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double m = i < npos ? (double)i : (double)(i - N);
    const double k = __dmul_rn(__dmul_rn(__dmul_rn(m, val), 2.0), M_PI);
    k1d[i] = k;
    k1t[i] = (T)k;
    double sn, cs;
    sincospi(2.0 * i / N, &sn, &cs);
    tw[i] = mkc<C>(cs, -sn);
  }
  __syncthreads();
  const double cutoff = __dmul_rn(2.0 / 3.0, __ddiv_rn(__dmul_rn(M_PI, (double)N), L));
  for (int ix = threadIdx.x; ix < N; ix += blockDim.x) {
    const double kx2 = __dmul_rn(k1d[ix], k1d[ix]);
    RowTab rt;
    rt.dmax = -1;
    rt.dragmax = -1;
    for (int my = 0; my <= H; ++my) {
      const double ky = k1d[my];
      if (__dsqrt_rn(__dadd_rn(kx2, __dmul_rn(ky, ky))) < cutoff) rt.dmax = my;
    }
    rt.pos_lo = 1; rt.pos_hi = 0; rt.neg_lo = 1; rt.neg_hi = 0;
    rt.row_start = 0;
    rt.pad = 0;
    rows[ix] = rt;
  }
  if (threadIdx.x == 0) *status = 0u;
}

template <typename T>
cudaError_t noalloc_tables(int N, double L, unsigned char* base, size_t o_k1d, size_t o_k1t, size_t o_tw,
                           size_t o_rows, size_t o_status, cudaStream_t st) {
  k_noalloc_tables<T><<<1, 256, 0, st>>>(N, L, (double*)(base + o_k1d), (T*)(base + o_k1t),
                                         (typename Cplx<T>::type*)(base + o_tw), (RowTab*)(base + o_rows),
                                         (unsigned*)(base + o_status));
  return cudaGetLastError();
}

}  // namespace

extern "C" int sqg_rhs_noalloc(const sqg_desc* desc, const void* theta, void* rhs, void* stream) {
  if (!desc || !theta || !rhs) return fail(SQG_ERR_INVALID, "null argument");
  const sqg_desc& d = *desc;
  if (d.N < 8 || d.N > SQG_NOALLOC_MAX_N || (d.N & (d.N - 1)) != 0)
    return fail(SQG_ERR_INVALID, "sqg_rhs_noalloc: N must be a power of two in [8, " +
                                     std::to_string(SQG_NOALLOC_MAX_N) + "] (static scratch of " +
                                     std::to_string(SQG_NOALLOC_SCRATCH_BYTES >> 20) + " MiB), got " +
                                     std::to_string(d.N));
  if (!(d.alpha >= -2 && d.alpha <= 2)) return fail(SQG_ERR_INVALID, "alpha must be in [-2, 2], got " + std::to_string(d.alpha));
  if (d.p != 2 && d.p != 4 && d.p != 8) return fail(SQG_ERR_INVALID, "p must be 2, 4, or 8, got " + std::to_string(d.p));
  if (d.precision != SQG_F64 && d.precision != SQG_F32) return fail(SQG_ERR_INVALID, "bad precision");
  if (!(d.L > 0)) return fail(SQG_ERR_INVALID, "L must be positive");
  int log2n = 0;
  while ((1 << log2n) < d.N) ++log2n;
  // The device address of the static array on the current device.  In host
  // code the array's name is only a host-side stand-in, never a device
  // address.  It is looked up on every call (a host-side table lookup once
  // the module is loaded), so no per-device cache can race between host
  // threads or go stale after a cudaDeviceReset; the first call on a device
  // loads the module and belongs before any stream capture.
  void* scratch = nullptr;
  SQG_CUDA(cudaGetSymbolAddress(&scratch, g_noalloc_scratch));
  // A plan that lives on the stack and points into the static scratch
  // (value-initialised: every offset and flag not set below is zero).
  sqg_plan pl{};
  pl.d = d;
  pl.d.has_damping = 0;
  pl.d.has_ring = 0;
  pl.d.n_scalars = 0;
  pl.N = d.N;
  pl.H = d.N / 2;
  pl.log2N = log2n;
  pl.csize = d.precision == SQG_F64 ? 16 : 8;
  pl.akind = alpha_kind(d.alpha);
  const size_t N = d.N, cs = pl.csize, half = (N / 2 + 1) * N * cs;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o += align256(bytes); return r; };
  pl.off_k1d = take(N * sizeof(double));
  pl.off_k1t = take(N * cs / 2);
  pl.off_tw = take(N * cs);
  pl.off_rows = take(N * sizeof(RowTab));
  pl.off_status = take(sizeof(unsigned));
  pl.off_ringF = pl.off_status;
  pl.off_xh = take(4 * half);
  pl.off_jh = take(half);
  pl.off_acc = pl.off_stage = pl.off_xh;  // unused by the RHS passes
  if (o > SQG_NOALLOC_SCRATCH_BYTES) return fail(SQG_ERR_INVALID, "sqg_rhs_noalloc: scratch too small");
  pl.ws = (unsigned char*)scratch;
  pl.ws_bytes = SQG_NOALLOC_SCRATCH_BYTES;
  pl.ready = true;
  cudaStream_t st = (cudaStream_t)stream;
  if (d.precision == SQG_F64) {
    SQG_CUDA(noalloc_tables<double>(pl.N, d.L, pl.ws, pl.off_k1d, pl.off_k1t, pl.off_tw, pl.off_rows, pl.off_status, st));
    SQG_CUDA(set_attrs_p<double>(log2n));
  } else {
    SQG_CUDA(noalloc_tables<float>(pl.N, d.L, pl.ws, pl.off_k1d, pl.off_k1t, pl.off_tw, pl.off_rows, pl.off_status, st));
    SQG_CUDA(set_attrs_p<float>(log2n));
  }
  int rc = run_p1(&pl, theta, FM_THETA, nullptr, st);
  if (rc != SQG_OK) return rc;
  KP kp = make_kp(&pl, 0.0);
  kp.ring_on = 0;
  ColArgs ca = base_col(&pl);
  SQG_CUDA(launch_col(&pl, kp, ca, st));
  RowArgs ra = base_row(&pl);
  ra.rmode = RM_RHS;
  ra.stage = 1;
  ra.th_n = theta;
  ra.rhs_out = rhs;
  ra.do_p1 = 0;
  SQG_CUDA(launch_row(&pl, kp, ra, st));
  return SQG_OK;
}

// ---------------------------------------------------------------------------
// Batched ensembles: every member of a batch has the same N and precision
// (one size class); alpha and the passive scalars vary per member.  One
// launch advances all members through a pass (member = blockIdx.y); a whole
// ensemble step is captured once in a CUDA graph and replayed.
// ---------------------------------------------------------------------------
struct sqg_batch {
  sqg_desc d;  // common physics: N, precision, scheme, p, nu_p, L, damping
  int N, H, log2N, M, S;
  size_t csize;
  std::vector<sqg_member> mem;
  std::vector<int> scal_member, scal_slot;  // scalar batch entry -> (member, slot)
  sqg_plan tables;                           // grid tables (a plan without per-field buffers)
  unsigned char* ws = nullptr;
  size_t ws_bytes = 0, off_tab = 0, off_member = 0, member_stride = 0, off_scalar = 0, scalar_stride = 0,
         off_args = 0, off_total = 0;
  // offsets inside a member block / scalar block
  size_t m_acc, m_stage, m_xh, m_jh, m_uv, s_acc, s_stage, s_xs, s_js;
  // device argument arrays
  KP* d_kp = nullptr;            // [M]
  KP* d_kps = nullptr;           // [S]
  RowArgs* d_p1 = nullptr;       // [M]
  ColArgs* d_col = nullptr;      // [M]
  RowArgs* d_row = nullptr;      // [4][M]
  ColArgs* d_vel = nullptr;      // [M]
  RowArgs* d_sp1 = nullptr;      // [S]
  ColArgs* d_scol = nullptr;     // [S]
  RowArgs* d_srow = nullptr;     // [4][S]
  ColArgs* d_scolv = nullptr;    // [S] first scalar stage with u, v from theta's spectra (multi-size path)
  RowArgs* d_srow4p = nullptr;   // [S] last scalar stage that also transforms s_{n+1} (multi-size path)
  double args_dt = -1.0;
  bool ready = false;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t cap = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int64_t launches = 0;
};

namespace {

template <typename T>
cudaError_t launch_row_batch_p(int log2n, const KP* kps, const RowArgs* as, int m, cudaStream_t st) {
  SQG_DISPATCH(log2n, launch_row_batch_t, kps, as, m, st);
}
template <typename T>
cudaError_t launch_col_batch_p(int log2n, const KP* kps, const ColArgs* as, int m, cudaStream_t st) {
  SQG_DISPATCH(log2n, launch_col_batch_t, kps, as, m, st);
}
template <typename T>
cudaError_t set_batch_attrs_p(int log2n) {
  SQG_DISPATCH(log2n, set_batch_attrs_t);
}

cudaError_t brow(sqg_batch* b, const KP* kps, const RowArgs* as, int m, cudaStream_t st) {
  if (m == 0) return cudaSuccess;
  b->launches++;
  return b->d.precision == SQG_F64 ? launch_row_batch_p<double>(b->log2N, kps, as, m, st)
                                   : launch_row_batch_p<float>(b->log2N, kps, as, m, st);
}
cudaError_t bcol(sqg_batch* b, const KP* kps, const ColArgs* as, int m, cudaStream_t st) {
  if (m == 0) return cudaSuccess;
  b->launches++;
  return b->d.precision == SQG_F64 ? launch_col_batch_p<double>(b->log2N, kps, as, m, st)
                                   : launch_col_batch_p<float>(b->log2N, kps, as, m, st);
}

// Builds and uploads every member's pass arguments for time step dt.
int batch_upload_args(sqg_batch* b, double dt, cudaStream_t st) {
  const int M = b->M, S = b->S;
  sqg_plan* tp = &b->tables;
  KP base = make_kp(tp, dt);
  base.ring_on = 0;
  base.n_ring = 0;
  std::vector<KP> kp(M), kps(std::max(S, 1));
  std::vector<RowArgs> p1(M), row(4 * M), sp1(std::max(S, 1)), srow(4 * std::max(S, 1));
  std::vector<ColArgs> col(M), vel(M), scol(std::max(S, 1)), scolv(std::max(S, 1));
  std::vector<RowArgs> srow4p(std::max(S, 1));
  const bool explicit_lin = b->d.scheme == SQG_EXPLICIT_RK4 &&
                            (b->d.nu_p != 0.0 || (b->d.has_damping && (b->d.mu != 0.0 || b->d.nu_damp != 0.0)));
  for (int i = 0; i < M; ++i) {
    unsigned char* mb = b->ws + b->off_member + (size_t)i * b->member_stride;
    kp[i] = base;
    kp[i].alpha = b->mem[i].alpha;
    kp[i].akind = alpha_kind(b->mem[i].alpha);
    RowArgs a;
    std::memset(&a, 0, sizeof(a));
    a.fmode = FM_THETA;
    a.xh = mb + b->m_xh;
    a.jh = mb + b->m_jh;
    a.acc = mb + b->m_acc;
    a.st_out = mb + b->m_stage;
    a.st_in = a.st_out;
    a.th_n = b->mem[i].theta;
    a.th_out = b->mem[i].theta;
    a.do_p1 = 1;
    p1[i] = a;
    p1[i].rmode = RM_P1;
    for (int s = 1; s <= 4; ++s) {
      RowArgs r = a;
      r.rmode = RM_STAGE;
      r.stage = s;
      r.stage_write = explicit_lin ? SW_FULL : SW_NONE;
      row[(s - 1) * M + i] = r;
    }
    ColArgs c;
    std::memset(&c, 0, sizeof(c));
    c.cmode = CM_THETA;
    c.xh = a.xh;
    c.jh = const_cast<void*>(a.jh);
    col[i] = c;
    ColArgs v = c;
    v.cmode = CM_VEL;
    v.out0 = mb + b->m_uv;
    v.out1 = nullptr;
    if (b->mem[i].n_scalars == 0) v.xh = nullptr;  // no work for this member
    vel[i] = v;
  }
  for (int k = 0; k < S; ++k) {
    const int i = b->scal_member[k], q = b->scal_slot[k];
    unsigned char* sb = b->ws + b->off_scalar + (size_t)k * b->scalar_stride;
    unsigned char* mb = b->ws + b->off_member + (size_t)i * b->member_stride;
    kps[k] = base;
    RowArgs a;
    std::memset(&a, 0, sizeof(a));
    a.fmode = FM_SCAL;
    a.xh = sb + b->s_xs;
    a.jh = sb + b->s_js;
    a.acc = sb + b->s_acc;
    a.st_out = sb + b->s_stage;
    a.st_in = a.st_out;
    a.th_n = b->mem[i].scalars[q];
    a.th_out = b->mem[i].scalars[q];
    a.kappa = b->mem[i].kappa[q];
    a.do_p1 = 1;
    sp1[k] = a;
    sp1[k].rmode = RM_P1;
    const bool sexp = b->d.scheme == SQG_EXPLICIT_RK4 && a.kappa != 0.0;
    for (int s = 1; s <= 4; ++s) {
      RowArgs r = a;
      r.rmode = RM_STAGE;
      r.stage = s;
      r.do_p1 = s < 4 ? 1 : 0;
      r.stage_write = sexp ? SW_FULL : SW_NONE;
      srow[(s - 1) * S + k] = r;
    }
    ColArgs c;
    std::memset(&c, 0, sizeof(c));
    c.cmode = CM_SCAL;
    c.xh = a.xh;
    c.jh = const_cast<void*>(a.jh);
    c.uv = mb + b->m_uv;
    scol[k] = c;
    // multi-size path: stage 1 transforms theta's u, v itself (its first
    // scalar writes u + i v for stages 2-4), and stage 4 also transforms
    // s_{n+1} for the next step
    ColArgs cv = c;
    cv.cmode = CM_SCALV;
    cv.xh = mb + b->m_xh;
    cv.xh2 = a.xh;
    cv.out0 = q == 0 ? mb + b->m_uv : nullptr;
    scolv[k] = cv;
    srow4p[k] = srow[3 * std::max(S, 1) + k];
    srow4p[k].do_p1 = 1;
  }
  auto up = [&](void* dst, const void* src, size_t n) {
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);
  };
  SQG_CUDA(up(b->d_kp, kp.data(), M * sizeof(KP)));
  SQG_CUDA(up(b->d_p1, p1.data(), M * sizeof(RowArgs)));
  SQG_CUDA(up(b->d_row, row.data(), 4 * M * sizeof(RowArgs)));
  SQG_CUDA(up(b->d_col, col.data(), M * sizeof(ColArgs)));
  SQG_CUDA(up(b->d_vel, vel.data(), M * sizeof(ColArgs)));
  if (S > 0) {
    SQG_CUDA(up(b->d_kps, kps.data(), S * sizeof(KP)));
    SQG_CUDA(up(b->d_sp1, sp1.data(), S * sizeof(RowArgs)));
    SQG_CUDA(up(b->d_srow, srow.data(), 4 * S * sizeof(RowArgs)));
    SQG_CUDA(up(b->d_scol, scol.data(), S * sizeof(ColArgs)));
    SQG_CUDA(up(b->d_scolv, scolv.data(), S * sizeof(ColArgs)));
    SQG_CUDA(up(b->d_srow4p, srow4p.data(), S * sizeof(RowArgs)));
  }
  SQG_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
  b->args_dt = dt;
  return SQG_OK;
}

// One ensemble step after the theta P1 pass of the step's input.
int batch_step_launches(sqg_batch* b, cudaStream_t st) {
  const int M = b->M, S = b->S;
  for (int s = 1; s <= 4; ++s) {
    SQG_CUDA(bcol(b, b->d_kp, b->d_col, M, st));
    SQG_CUDA(brow(b, b->d_kp, b->d_row + (size_t)(s - 1) * M, M, st));
  }
  if (S > 0) {
    // u + i v of theta_{n+1} from the stage-4 transforms, then the scalars
    SQG_CUDA(bcol(b, b->d_kp, b->d_vel, M, st));
    SQG_CUDA(brow(b, b->d_kps, b->d_sp1, S, st));
    for (int s = 1; s <= 4; ++s) {
      SQG_CUDA(bcol(b, b->d_kps, b->d_scol, S, st));
      SQG_CUDA(brow(b, b->d_kps, b->d_srow + (size_t)(s - 1) * S, S, st));
    }
  }
  return SQG_OK;
}

}  // namespace

extern "C" {

int sqg_batch_create(const sqg_desc* desc, int32_t n_members, const sqg_member* members, sqg_batch** out) {
  if (!desc || !members || !out || n_members <= 0) return fail(SQG_ERR_INVALID, "bad batch arguments");
  sqg_desc d = *desc;
  d.has_ring = 0;
  d.n_scalars = 0;
  sqg_plan* tp = nullptr;
  int rc = sqg_plan_create(&d, &tp);
  if (rc != SQG_OK) return rc;
  sqg_batch* b = new sqg_batch();
  b->tables = *tp;
  b->tables.off_total = b->tables.off_acc;  // the batch keeps only the grid tables of the plan
  sqg_plan_destroy(tp);
  b->d = d;
  b->N = d.N;
  b->H = d.N / 2;
  b->log2N = b->tables.log2N;
  b->csize = b->tables.csize;
  b->M = n_members;
  b->mem.assign(members, members + n_members);
  for (int i = 0; i < n_members; ++i) {
    const sqg_member& m = members[i];
    if (!m.theta) { delete b; return fail(SQG_ERR_INVALID, "member theta is null"); }
    if (!(m.alpha >= -2 && m.alpha <= 2)) { delete b; return fail(SQG_ERR_INVALID, "alpha must be in [-2, 2]"); }
    if (m.n_scalars < 0 || m.n_scalars > SQG_MAX_SCALARS) { delete b; return fail(SQG_ERR_INVALID, "n_scalars out of range"); }
    for (int q = 0; q < m.n_scalars; ++q) {
      if (!m.scalars[q]) { delete b; return fail(SQG_ERR_INVALID, "member scalar is null"); }
      b->scal_member.push_back(i);
      b->scal_slot.push_back(q);
    }
  }
  b->S = (int)b->scal_member.size();
  const size_t N = b->N, cs = b->csize, full = N * N * cs, half = (N / 2 + 1) * N * cs;
  auto al = [](size_t x) { return align256(x); };
  b->m_acc = 0;
  b->m_stage = al(full);
  b->m_xh = b->m_stage + al(full);
  b->m_jh = b->m_xh + al(4 * half);
  b->m_uv = b->m_jh + al(half);
  b->member_stride = b->m_uv + al(full);
  b->s_acc = 0;
  b->s_stage = al(full);
  b->s_xs = b->s_stage + al(full);
  b->s_js = b->s_xs + al(2 * half);
  b->scalar_stride = b->s_js + al(half);
  b->off_tab = 0;
  b->off_member = al(b->tables.off_acc);  // grid tables come first, as in a plan
  b->off_scalar = b->off_member + (size_t)b->M * b->member_stride;
  b->off_args = b->off_scalar + (size_t)b->S * b->scalar_stride;
  const size_t Sx = std::max(b->S, 1);
  b->off_total = b->off_args + al(b->M * sizeof(KP)) + al(Sx * sizeof(KP)) + al(b->M * sizeof(RowArgs)) +
                 al(b->M * sizeof(ColArgs)) + al(4 * b->M * sizeof(RowArgs)) + al(b->M * sizeof(ColArgs)) +
                 al(Sx * sizeof(RowArgs)) + al(Sx * sizeof(ColArgs)) + al(4 * Sx * sizeof(RowArgs)) +
                 al(Sx * sizeof(ColArgs)) + al(Sx * sizeof(RowArgs));
  *out = b;
  return SQG_OK;
}

int sqg_batch_workspace_bytes(const sqg_batch* b, size_t* bytes) {
  if (!b || !bytes) return fail(SQG_ERR_INVALID, "null argument");
  *bytes = b->off_total;
  return SQG_OK;
}

int sqg_batch_set_workspace(sqg_batch* b, void* ws, size_t bytes, void* stream) {
  if (!b) return fail(SQG_ERR_INVALID, "null batch");
  if (!ws || bytes < b->off_total) return fail(SQG_ERR_WORKSPACE, "workspace missing or too small");
  // grid tables: the first bytes of the workspace, as a plan lays them out
  int rc = sqg_plan_set_workspace(&b->tables, ws, b->tables.off_acc, stream);
  if (rc != SQG_OK) return rc;
  b->ws = (unsigned char*)ws;
  b->ws_bytes = bytes;
  size_t o = b->off_args;
  auto take = [&](size_t n) { unsigned char* p = b->ws + o; o += align256(n); return p; };
  const size_t Sx = std::max(b->S, 1);
  b->d_kp = (KP*)take(b->M * sizeof(KP));
  b->d_kps = (KP*)take(Sx * sizeof(KP));
  b->d_p1 = (RowArgs*)take(b->M * sizeof(RowArgs));
  b->d_col = (ColArgs*)take(b->M * sizeof(ColArgs));
  b->d_row = (RowArgs*)take(4 * b->M * sizeof(RowArgs));
  b->d_vel = (ColArgs*)take(b->M * sizeof(ColArgs));
  b->d_sp1 = (RowArgs*)take(Sx * sizeof(RowArgs));
  b->d_scol = (ColArgs*)take(Sx * sizeof(ColArgs));
  b->d_srow = (RowArgs*)take(4 * Sx * sizeof(RowArgs));
  b->d_scolv = (ColArgs*)take(Sx * sizeof(ColArgs));
  b->d_srow4p = (RowArgs*)take(Sx * sizeof(RowArgs));
  if (b->d.precision == SQG_F64) { SQG_CUDA(set_batch_attrs_p<double>(b->log2N)); }
  else { SQG_CUDA(set_batch_attrs_p<float>(b->log2N)); }
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  b->args_dt = -1.0;
  b->ready = true;
  return SQG_OK;
}

int sqg_batch_multistep(sqg_batch* b, int32_t n_steps, double dt, int32_t use_graph, void* stream) {
  if (!b) return fail(SQG_ERR_INVALID, "null batch");
  if (!b->ready) return fail(SQG_ERR_WORKSPACE, "workspace not set (call sqg_batch_set_workspace)");
  if (n_steps < 0) return fail(SQG_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return SQG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (b->args_dt != dt) {
    if ((rc = batch_upload_args(b, dt, st)) != SQG_OK) return rc;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  }
  b->launches = 0;
  // theta P1 of every member's input state
  SQG_CUDA(brow(b, b->d_kp, b->d_p1, b->M, st));
  if (!use_graph) {
    for (int n = 0; n < n_steps; ++n)
      if ((rc = batch_step_launches(b, st)) != SQG_OK) return rc;
    return SQG_OK;
  }
  if (!b->cap) {
    SQG_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    SQG_CUDA(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming));
    SQG_CUDA(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming));
  }
  if (!b->graph) {
    cudaGraph_t g;
    SQG_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int64_t saved = b->launches;
    rc = batch_step_launches(b, b->cap);
    cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
    const int64_t per_step = b->launches - saved;
    b->launches = saved;
    if (rc != SQG_OK) return rc;
    if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
    b->tables.launches = per_step;  // launches in one replay
  }
  SQG_CUDA(cudaEventRecord(b->ev_in, st));
  SQG_CUDA(cudaStreamWaitEvent(b->cap, b->ev_in, 0));
  for (int n = 0; n < n_steps; ++n) {
    SQG_CUDA(cudaGraphLaunch(b->graph, b->cap));
    b->launches += b->tables.launches;
  }
  SQG_CUDA(cudaEventRecord(b->ev_out, b->cap));
  SQG_CUDA(cudaStreamWaitEvent(st, b->ev_out, 0));
  return SQG_OK;
}

int sqg_batch_last_launch_count(const sqg_batch* b, int64_t* n) {
  if (!b || !n) return fail(SQG_ERR_INVALID, "null argument");
  *n = b->launches;
  return SQG_OK;
}

int sqg_batch_destroy(sqg_batch* b) {
  if (!b) return SQG_OK;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  b->tables.graph_exec = nullptr;
  b->tables.cap_stream = nullptr;
  b->tables.ev_in = b->tables.ev_out = nullptr;
  delete b;
  return SQG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-size ensembles: the members of several batches (size classes
// N = 128, 256, 512) advance in one launch per pass of every RK stage.  The
// scalars run one step behind theta in the same launches: the scalar step
// that needs u, v of theta_{n+1} (frozen over its stages) runs beside theta's
// step n+2, whose first column pass reads the half spectra of theta_{n+1};
// the scalar's first column pass transforms u and v from them.  multistep(n)
// is: the input transforms of theta_0 and s_0 (one launch), theta's first
// step alone, n - 1 fused steps (replayed from one CUDA graph) and the last
// scalar step alone -- the same arithmetic as stepping theta and then the
// scalars, step after step.
// ---------------------------------------------------------------------------
struct sqg_ensemble {
  std::vector<sqg_batch*> cls;
  int precision = SQG_F32;
  cudaGraphExec_t graph = nullptr;
  double graph_dt = -1.0;
  cudaStream_t cap = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int64_t launches = 0;
};

namespace {

enum { EK_P1 = 0, EK_COL = 1, EK_ROW = 2 };

// Segments of one multi-size launch: kind EK_*, RK stage s (1..4), which
// entities take part, and whether the scalars run pipelined (their first
// stage transforms u, v; their last stage also transforms s_{n+1}).
int ens_segments(const sqg_ensemble* e, int kind, int s, bool theta, bool scalars, MultiArgs& ma) {
  std::memset(&ma, 0, sizeof(ma));
  int blocks = 0;
  auto add = [&](int log2n, int tiles, int count, const KP* kps, const void* args) {
    if (count <= 0) return;
    MultiSeg& g = ma.seg[ma.nseg++];
    g.start = blocks;
    g.tiles = tiles;
    g.log2n = log2n;
    g.kps = kps;
    g.args = args;
    blocks += tiles * count;
  };
  const bool f64 = e->precision == SQG_F64;
  for (int pass = 0; pass < 2; ++pass) {  // theta segments first, then the scalars
    for (sqg_batch* b : e->cls) {
      const int L = b->log2N;
      const int tiles = kind == EK_COL ? (f64 ? multi_col_tiles<double>(L) : multi_col_tiles<float>(L))
                                       : (f64 ? multi_row_tiles<double>(L) : multi_row_tiles<float>(L));
      if (pass == 0 && theta) {
        const void* args = kind == EK_P1 ? (const void*)b->d_p1
                           : kind == EK_COL ? (const void*)b->d_col : (const void*)(b->d_row + (size_t)(s - 1) * b->M);
        add(L, tiles, b->M, b->d_kp, args);
      }
      if (pass == 1 && scalars && b->S > 0) {
        const void* args;
        if (kind == EK_P1) args = b->d_sp1;
        else if (kind == EK_COL) args = s == 1 ? (const void*)b->d_scolv : (const void*)b->d_scol;
        else args = (s == 4 && theta) ? (const void*)b->d_srow4p : (const void*)(b->d_srow + (size_t)(s - 1) * b->S);
        add(L, tiles, b->S, b->d_kps, args);
      }
    }
  }
  return blocks;
}

cudaError_t ens_launch(sqg_ensemble* e, int kind, int s, bool theta, bool scalars, cudaStream_t st) {
  MultiArgs ma;
  const int blocks = ens_segments(e, kind, s, theta, scalars, ma);
  if (blocks == 0) return cudaSuccess;
  e->launches++;
  const bool f64 = e->precision == SQG_F64;
  if (kind == EK_COL) return f64 ? launch_col_multi<double>(ma, blocks, st) : launch_col_multi<float>(ma, blocks, st);
  return f64 ? launch_row_multi<double>(ma, blocks, st) : launch_row_multi<float>(ma, blocks, st);
}

// One RK step: the four stages of the given entities.
cudaError_t ens_step(sqg_ensemble* e, bool theta, bool scalars, cudaStream_t st) {
  for (int s = 1; s <= 4; ++s) {
    cudaError_t c = ens_launch(e, EK_COL, s, theta, scalars, st);
    if (c != cudaSuccess) return c;
    if ((c = ens_launch(e, EK_ROW, s, theta, scalars, st)) != cudaSuccess) return c;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

int sqg_ensemble_create(sqg_batch* const* classes, int32_t n_classes, sqg_ensemble** out) {
  if (!classes || !out || n_classes < 1 || n_classes > 3) return fail(SQG_ERR_INVALID, "1 to 3 size classes");
  sqg_ensemble* e = new sqg_ensemble();
  for (int i = 0; i < n_classes; ++i) {
    sqg_batch* b = classes[i];
    std::string why;
    if (!b) why = "null batch";
    else if (!b->ready) why = "batch workspace not set";
    else if (b->log2N < kMultiLo || b->log2N > kMultiHi) why = "multi-size launches serve N = 128, 256, 512";
    else if (i > 0 && b->d.precision != classes[0]->d.precision) why = "all classes need the same precision";
    else if (i > 0 && b->d.scheme != classes[0]->d.scheme) why = "all classes need the same time scheme";
    for (int k = 0; k < i && why.empty(); ++k)
      if (classes[k]->log2N == b->log2N) why = "each size class at most once";
    if (!why.empty()) { delete e; return fail(SQG_ERR_INVALID, "sqg_ensemble_create: " + why); }
    e->cls.push_back(b);
  }
  e->precision = classes[0]->d.precision;
  cudaError_t c = e->precision == SQG_F64 ? set_multi_attrs<double>() : set_multi_attrs<float>();
  if (c != cudaSuccess) { delete e; return fail(SQG_ERR_CUDA, std::string("multi-size kernels: ") + cudaGetErrorString(c)); }
  *out = e;
  return SQG_OK;
}

int sqg_ensemble_multistep(sqg_ensemble* e, int32_t n_steps, double dt, int32_t use_graph, void* stream) {
  if (!e) return fail(SQG_ERR_INVALID, "null ensemble");
  if (n_steps < 0) return fail(SQG_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return SQG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  bool any_scalars = false;
  for (sqg_batch* b : e->cls) {
    if (b->args_dt != dt) {
      if ((rc = batch_upload_args(b, dt, st)) != SQG_OK) return rc;
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    }
    any_scalars |= b->S > 0;
  }
  if (e->graph && e->graph_dt != dt) { cudaGraphExecDestroy(e->graph); e->graph = nullptr; }
  e->launches = 0;
  // input transforms of theta_0 and s_0, then theta's first step alone
  SQG_CUDA(ens_launch(e, EK_P1, 1, true, true, st));
  SQG_CUDA(ens_step(e, true, false, st));
  if (n_steps > 1) {
    if (!use_graph) {
      for (int n = 1; n < n_steps; ++n) SQG_CUDA(ens_step(e, true, true, st));
    } else {
      if (!e->cap) {
        SQG_CUDA(cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking));
        SQG_CUDA(cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming));
        SQG_CUDA(cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming));
      }
      int64_t per = 0;
      if (!e->graph) {
        cudaGraph_t g;
        SQG_CUDA(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal));
        const int64_t saved = e->launches;
        cudaError_t c = ens_step(e, true, true, e->cap);
        cudaError_t ce = cudaStreamEndCapture(e->cap, &g);
        per = e->launches - saved;
        e->launches = saved;
        if (c != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(c));
        if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return fail(SQG_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
        e->graph_dt = dt;
      } else {
        MultiArgs ma;
        for (int s = 1; s <= 4; ++s) {
          per += ens_segments(e, EK_COL, s, true, true, ma) > 0;
          per += ens_segments(e, EK_ROW, s, true, true, ma) > 0;
        }
      }
      SQG_CUDA(cudaEventRecord(e->ev_in, st));
      SQG_CUDA(cudaStreamWaitEvent(e->cap, e->ev_in, 0));
      for (int n = 1; n < n_steps; ++n) {
        SQG_CUDA(cudaGraphLaunch(e->graph, e->cap));
        e->launches += per;
      }
      SQG_CUDA(cudaEventRecord(e->ev_out, e->cap));
      SQG_CUDA(cudaStreamWaitEvent(st, e->ev_out, 0));
    }
  }
  // the scalars' last step (with u, v of the final theta)
  if (any_scalars) SQG_CUDA(ens_step(e, false, true, st));
  return SQG_OK;
}

int sqg_ensemble_last_launch_count(const sqg_ensemble* e, int64_t* n) {
  if (!e || !n) return fail(SQG_ERR_INVALID, "null argument");
  *n = e->launches;
  return SQG_OK;
}

int sqg_ensemble_destroy(sqg_ensemble* e) {
  if (!e) return SQG_OK;
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->cap) cudaStreamDestroy(e->cap);
  if (e->ev_in) cudaEventDestroy(e->ev_in);
  if (e->ev_out) cudaEventDestroy(e->ev_out);
  delete e;
  return SQG_OK;
}

}  // extern "C"
