/*
 * sqg.h -- C ABI of libsqg, the B200 (sm_100a) kernels behind pygsquig_b200.
 *
 * One plan = one doubly periodic N x N grid with fixed physics (alpha,
 * hyperviscosity, damping, ring forcing, passive scalars), precision and time
 * scheme.  All device memory is owned by the caller: the plan reports how many
 * workspace bytes it needs, the caller allocates them (e.g. a torch uint8
 * tensor) and hands the pointer over once with sqg_plan_set_workspace.  No
 * entry point allocates device memory.  Every call is asynchronous on the
 * given CUDA stream (NULL = legacy default stream) and returns an sqg_status;
 * sqg_last_error_string() describes the last failure of the calling thread.
 *
 * Spectra are full N x N complex arrays (complex128 for SQG_F64, complex64
 * for SQG_F32), row-major, axis 0 = kx, axis 1 = ky -- the layout of the
 * reference's theta_hat (pygsquig/core/grid.py:90-95, solver.py:96-124).
 * Physical fields are N x N real arrays, axis 0 = x.
 *
 * Threading: a plan is not thread-safe; distinct plans are independent.
 */
#ifndef SQG_H
#define SQG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SQG_MAX_SCALARS 4

typedef enum {
  SQG_OK = 0,
  SQG_ERR_INVALID = 1,   /* bad argument or unsupported size (-> ValueError) */
  SQG_ERR_CUDA = 2,      /* CUDA runtime error */
  SQG_ERR_NONFINITE = 3, /* non-finite value produced (-> NumericalError) */
  SQG_ERR_WORKSPACE = 4, /* workspace missing or too small */
  SQG_ERR_STATE = 5      /* calls made in an invalid order */
} sqg_status;

typedef enum { SQG_F64 = 0, SQG_F32 = 1 } sqg_precision;

/* SQG_EXPLICIT_RK4: classic RK4 with every term in the right-hand side
 *   (pygsquig/core/time_integrator.py:14-36) -- the reference scheme.
 * SQG_IF_RK4: integrating-factor RK4; the diagonal terms (solver and damping
 *   hyperviscosity, large-scale drag, scalar diffusion) go through
 *   exp(L dt / 2) evaluated in float64.  Extension for stiff hyperviscosity. */
typedef enum { SQG_EXPLICIT_RK4 = 0, SQG_IF_RK4 = 1 } sqg_scheme;

typedef struct sqg_desc {
  int32_t N;          /* power of two, 8 <= N <= 4096 */
  int32_t precision;  /* sqg_precision */
  int32_t scheme;     /* sqg_scheme */
  int32_t p;          /* solver hyperviscosity order: 2, 4 or 8 */
  double L;           /* domain size */
  double alpha;       /* gSQG exponent, -2 <= alpha <= 2 */
  double nu_p;        /* solver hyperviscosity, -nu_p k2^(p/2) (operators.py:185-207) */
  /* CombinedDamping carried by the plan (pygsquig/forcing/damping.py:49-92) */
  int32_t has_damping;
  int32_t p_damp;
  double mu;          /* large-scale drag on |k| < kf_damp / 2 */
  double kf_damp;
  double nu_damp;     /* damping hyperviscosity (adds to nu_p, as the reference does) */
  /* RingForcing carried by the plan (pygsquig/forcing/ring_forcing.py:16-170) */
  int32_t has_ring;
  int32_t reserved0;
  double ring_kf, ring_dk, ring_epsilon, ring_tau_f, ring_amplitude;
  /* passive scalars (pygsquig/scalars/passive_scalar.py:24-258) */
  int32_t n_scalars;
  int32_t reserved1;
  double kappa[SQG_MAX_SCALARS];
  int32_t mean_gradient[SQG_MAX_SCALARS]; /* 1: source S = -(gx u + gy v) */
  double grad_x[SQG_MAX_SCALARS];
  double grad_y[SQG_MAX_SCALARS];
} sqg_desc;

typedef struct sqg_plan sqg_plan;

/* Buffers inside the workspace that the host may view (sqg_plan_buffer). */
typedef enum {
  SQG_BUF_STAGE = 0,      /* N x N complex: stage input theta_s of the last stage */
  SQG_BUF_UV = 1,         /* N x N complex u + i v (physical) at the new time, column-pair-major:
                             (x, y) at element ((y / 2) N + x) 2 + (y mod 2) */
  SQG_BUF_RING_FORCE = 2, /* n_ring complex128: ring forcing of the last stage (scaled) */
  SQG_BUF_STATUS = 3      /* uint32 status flags */
} sqg_buffer;

/* Replaces gSQGSolver.__init__ validation + make_grid (solver.py:75-94,
 * grid.py:72-107), CombinedDamping.__init__ (damping.py:49-73) and
 * RingForcing.__init__/_get_forcing_mask (ring_forcing.py:31-76). */
int sqg_plan_create(const sqg_desc* desc, sqg_plan** out);
int sqg_plan_destroy(sqg_plan* plan);
int sqg_plan_workspace_bytes(const sqg_plan* plan, size_t* bytes);
/* Takes the caller's device workspace and uploads the grid tables into it. */
int sqg_plan_set_workspace(sqg_plan* plan, void* workspace, size_t bytes, void* stream);
int sqg_plan_buffer(const sqg_plan* plan, int32_t which, size_t* offset, size_t* bytes);

/* Ring modes in row-major order of |sqrt(k2) - kf| <= dk/2
 * (ring_forcing.py:64-76); phases passed to the step calls use this order. */
int sqg_ring_mode_count(const sqg_plan* plan, int32_t* n_ring);
int sqg_ring_modes(const sqg_plan* plan, int32_t* ix, int32_t* iy);

/* Split forcing (an extension for coarse solves whose step is larger than
 * the step the forcing statistics were set with): n_sub forcing-only RK4
 * sub-steps of length dt_sub on the ring modes of theta_hat, in place, each
 * with its own row of phases (device float64[n_sub][n_ring]).  Each sub-step
 * is the RK4 step of d theta/dt = s(<theta F>) F with the reference's rescale
 * s(r) = eps / r (ring_forcing.py:151-170), computed exactly through the
 * linearity of <theta F> in theta.  White-in-time forcing only (tau_f = 0). */
int sqg_ring_substeps(sqg_plan* plan, void* theta_hat, int32_t n_sub, double dt_sub, const double* phases,
                      void* stream);

/* Launch shapes of the transform passes (an extension; the reference has no
 * kernels to shape).  The row pass runs rpc row pairs per CTA and the column
 * pass np column pairs per CTA, each a power-of-two divisor of a compiled
 * maximum (0 selects the maximum).  The shape changes speed only: every
 * transform is computed the same way, so results are bit-identical across
 * shapes.  sqg_plan_autotune times the passes of one right-hand side for
 * every shape on the plan's own workspace (which must be set) and keeps the
 * fastest; it synchronises the stream. */
int sqg_plan_shape(const sqg_plan* plan, int32_t* rpc, int32_t* np, int32_t* max_rpc, int32_t* max_np);
int sqg_plan_set_shape(sqg_plan* plan, int32_t rpc, int32_t np);
int sqg_plan_autotune(sqg_plan* plan, int32_t reps, void* stream);

/* Core RHS -fft2(jacobian) + hyperviscosity(nu_p) of theta_hat
 * (replaces _compute_core_rhs, pygsquig/core/solver.py:28-58). */
int sqg_rhs(sqg_plan* plan, const void* theta_hat, void* rhs, void* stream);

/* No counterpart in the reference.  sqg_rhs for callers that cannot
 * allocate device memory -- for example a host application that reserves all
 * device memory up front through its own allocator, or a latency-critical loop
 * in which cudaMalloc/cudaFree are not allowed because they can synchronise
 * the device.  It takes a descriptor instead of a plan and needs no
 * workspace: the grid tables and intermediate fields live in a static device
 * array of SQG_NOALLOC_SCRATCH_BYTES (3 MiB) that every GPU loading the
 * library keeps until the process exits.  Limit: N <= SQG_NOALLOC_MAX_N (256),
 * larger N is rejected with SQG_ERR_INVALID.  Each call looks up the array's
 * device address on the current device (cudaGetSymbolAddress); the first
 * call on a device also loads the library's device code there, so make that
 * first call before any stream capture.  Every call rewrites the whole
 * array, so calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Only N, L, alpha,
 * nu_p, p and precision of the descriptor are used.  The twiddle table is
 * computed on the device here (on the host for a plan), so the result equals
 * sqg_rhs's to rounding, not bit for bit. */
#define SQG_NOALLOC_MAX_N 256
#define SQG_NOALLOC_SCRATCH_BYTES (3u << 20)
int sqg_rhs_noalloc(const sqg_desc* desc, const void* theta_hat, void* rhs, void* stream);

/* One RK4 step theta_out = step(theta_in) (replaces gSQGSolver.step with the
 * plan's forcing/damping, solver.py:182-214 + time_integrator.py:14-36).
 * ring_phases: device float64[n_ring] in [0, 2pi) (NULL if no ring forcing).
 * theta_out may equal theta_in. */
int sqg_step(sqg_plan* plan, const void* theta_in, void* theta_out, double dt,
             const double* ring_phases, void* stream);

/* n_steps RK4 steps in place (replaces gSQGSolverOptimized.multistep,
 * solver_optimized.py:168-199, extended with forcing/damping).
 * ring_phases: device float64[n_steps][n_ring] or NULL.  With use_graph != 0
 * one step is captured in a CUDA graph and replayed. */
int sqg_multistep(sqg_plan* plan, void* theta_hat, int32_t n_steps, double dt,
                  const double* ring_phases, int32_t use_graph, void* stream);

/* Generic stepping, for forcing/damping callables the plan does not carry:
 *   sqg_stage_begin(theta_in); then for s = 1..4:
 *     extra_s = f(theta_s)   (theta_s = theta_in for s = 1, else SQG_BUF_STAGE)
 *     sqg_stage(s, extra_s)
 * After stage 4 theta_out holds the new state.  extra may be NULL. */
int sqg_stage_begin(sqg_plan* plan, const void* theta_in, void* stream);
int sqg_stage(sqg_plan* plan, int32_t stage, const void* theta_in, void* theta_out,
              double dt, const void* extra_rhs, const double* ring_phases, void* stream);

/* The same stage with an extra tendency given in physical space: src is a
 * real N x N field of the plan precision, and the stage right-hand side is
 * -mask fft2(u.grad theta - src) + (linear terms, forcing): src is added to
 * the advective term inside the column pass and dealiased with it (a learned
 * subgrid closure enters the coarse solve this way).  Extension: the
 * reference adds forcing terms in spectral space only (solver.py:170-178). */
int sqg_stage_physical(sqg_plan* plan, int32_t stage, const void* theta_in, void* theta_out,
                       double dt, const void* src, const double* ring_phases, void* stream);

/* Velocity (u, v) in physical space (replaces compute_velocity_from_theta,
 * operators.py:159-181).  u and v: N x N real of the plan precision. */
int sqg_velocity(sqg_plan* plan, const void* theta_hat, void* u, void* v, void* stream);

/* Inverse transform Re ifft2 of a full spectrum (grid.py:127-138). */
int sqg_to_physical(sqg_plan* plan, const void* field_hat, void* field, void* stream);

/* Forward transform fft2 of a real N x N field (grid.py:110-124). */
int sqg_to_spectral(sqg_plan* plan, const void* field, void* field_hat, void* stream);

/* Solver hyperviscosity -nu_p k2^(p/2) theta_hat, zero at k = 0
 * (replaces hyperviscosity, operators.py:185-207). */
int sqg_hyperviscosity(sqg_plan* plan, const void* theta_hat, void* out, void* stream);

/* Mean of Re ifft2(a) * Re ifft2(b) (the <theta F> of ring_forcing.py:153-155
 * and the dissipation rates of damping.py:113-116); out: device float64[1]. */
int sqg_inner(sqg_plan* plan, const void* a_hat, const void* b_hat, double* out, void* stream);

/* Diagonal damping term of CombinedDamping(mu, kf_damp, nu_damp, p_damp)
 * (damping.py:75-92) applied to theta_hat: out = L_damp * theta_hat. */
int sqg_damping(sqg_plan* plan, const void* theta_hat, void* out, void* stream);

/* RingForcing.__call__ (ring_forcing.py:119-170): forcing spectrum for
 * theta_hat with the given phases, rescaled to <theta F> = epsilon. */
int sqg_ring_forcing(sqg_plan* plan, const void* theta_hat, const double* ring_phases,
                     double dt, void* out, void* stream);

/* Diagnostics, float64 on the device (out: device float64[SQG_DIAG_COUNT]):
 *  [0] total energy   1/2 sum k2^((a-2)/2)|th|^2 / N^2   (utils/diagnostics.py:171-190)
 *  [1] enstrophy      1/2 sum |k|^(2a) |th|^2            (utils/diagnostics.py:120-141)
 *  [2] kinetic energy 1/2 <u^2 + v^2>                    (solver.py:229-231)
 *  [3] 1/2 <theta^2>                                     (solver.py:233-234)
 *  [4] max |theta|                                       (solver.py:236-237)
 *  [5] palinstrophy                                      (utils/diagnostics.py:194-217) */
#define SQG_DIAG_COUNT 6
int sqg_diagnostics(sqg_plan* plan, const void* theta_hat, double* out, void* stream);

/* Maxima for adaptive time stepping (replace compute_max_velocity,
 * pygsquig/core/adaptive_timestep.py:59-68, and the max |theta_hat| of the
 * stability check, :288-305): out = device float64, NaN if any element is
 * not finite.  u, v: real N x N of the plan precision. */
int sqg_max_speed(sqg_plan* plan, const void* u, const void* v, double* out, void* stream);
int sqg_spectrum_absmax(sqg_plan* plan, const void* theta_hat, double* out, void* stream);

/* Shell energy spectrum E(k) (utils/diagnostics.py:31-84), n_bins =
 * min(N/4, 64) linear bins; out: device float64[n_bins]. */
int sqg_energy_spectrum(sqg_plan* plan, const void* theta_hat, double* out, void* stream);

/* Scalar variance <(s - <s>)^2> of a spectrum (scalars/diagnostics.py:156-168). */
int sqg_scalar_variance(sqg_plan* plan, const void* s_hat, double* out, void* stream);

/* Passive scalars (solver_with_scalars.py:131-178): after a theta step to
 * theta_new, advance every scalar one RK4 step with (u, v) of theta_new frozen
 * over the stages.  scalars_in/out: n_scalars pointers to N x N spectra. */
int sqg_scalars_step(sqg_plan* plan, const void* theta_new, const void* const* scalars_in,
                     void* const* scalars_out, double dt, void* stream);

/* Batched ensembles (replaces the pmap ensemble of multi_gpu.py:118-155 on
 * one GPU): members share N, precision, scheme and the solver/damping
 * physics of the descriptor; alpha and up to SQG_MAX_SCALARS passive scalars
 * (diffusivity kappa, no source) vary per member.  Every pass of an RK stage
 * is one launch over all members (member = blockIdx.y); sqg_batch_multistep
 * advances every member's state in place, replaying one captured CUDA graph
 * per step.  Each step updates theta first, then the member's scalars with
 * theta's new velocity frozen over the stages (solver_with_scalars.py:
 * 131-178).  Ring forcing is not carried by batches. */
typedef struct sqg_member {
  void* theta;                       /* N x N spectrum, advanced in place */
  double alpha;
  int32_t n_scalars;
  int32_t reserved;
  void* scalars[SQG_MAX_SCALARS];    /* N x N spectra, advanced in place */
  double kappa[SQG_MAX_SCALARS];
} sqg_member;
typedef struct sqg_batch sqg_batch;
int sqg_batch_create(const sqg_desc* desc, int32_t n_members, const sqg_member* members, sqg_batch** out);
int sqg_batch_workspace_bytes(const sqg_batch* batch, size_t* bytes);
int sqg_batch_set_workspace(sqg_batch* batch, void* workspace, size_t bytes, void* stream);
int sqg_batch_multistep(sqg_batch* batch, int32_t n_steps, double dt, int32_t use_graph, void* stream);
int sqg_batch_last_launch_count(const sqg_batch* batch, int64_t* launches);
int sqg_batch_destroy(sqg_batch* batch);

/* Multi-size ensembles (the pmap ensemble of multi_gpu.py:118-155, for
 * members of uneven resolution): the members of up to three batches of
 * distinct size classes N = 128, 256, 512 (same precision and scheme) advance
 * in ONE launch per pass of every RK stage -- eight launches per step for
 * theta and every scalar of every member.  The scalars run one step behind
 * theta inside the same launches (the scalar step that needs u, v of
 * theta_{n+1} runs beside theta's step n+2 and transforms u, v from the half
 * spectra that step reads), so sqg_ensemble_multistep(n) gives the same
 * states as n batch steps: theta first, then the scalars with theta's new
 * velocity (solver_with_scalars.py:131-178).  The batches keep owning the
 * member buffers; destroy the ensemble before them. */
typedef struct sqg_ensemble sqg_ensemble;
int sqg_ensemble_create(sqg_batch* const* classes, int32_t n_classes, sqg_ensemble** out);
int sqg_ensemble_multistep(sqg_ensemble* ensemble, int32_t n_steps, double dt, int32_t use_graph, void* stream);
int sqg_ensemble_last_launch_count(const sqg_ensemble* ensemble, int64_t* launches);
int sqg_ensemble_destroy(sqg_ensemble* ensemble);

/* Reads and clears the sticky status flags (bit 0: non-finite value seen;
 * bit 1: a column pass's TMA tile copies did not complete within its bounded
 * wait, so its results are not valid).  Synchronises the stream. */
int sqg_check_status(sqg_plan* plan, uint32_t* flags, void* stream);

/* Number of kernel launches the last sqg_step / sqg_multistep issued. */
int sqg_last_launch_count(const sqg_plan* plan, int64_t* launches);

/* Per-launch timing with CUDA events on the launching stream (instrumentation
 * for benchmarks; multistep then runs without its CUDA graph).  enable = 0
 * off, 1 one event pair around every launch, k > 1 every launch site issues
 * its pass k times back to back inside one event pair (the passes chained by
 * programmatic dependent launch as inside a step; the results of such a call
 * are not valid -- RK accumulators are updated k times -- and the next step
 * recomputes every buffer from its inputs; refused for OU ring forcing,
 * whose state the repeats would advance).  sqg_timing_read synchronises,
 * returns total milliseconds and launch counts per kind (0 theta row inverse
 * pass, 1 theta row stage pass with transforms, 2 theta column pass, 3 scalar
 * row stage pass, 4 scalar column pass, 5 other, 6 theta row stage pass
 * without transforms (last stage), 7 velocity row pass, 8 velocity column
 * pass, 9 scalar row inverse pass) and clears the record. */
int sqg_set_timing(sqg_plan* plan, int32_t enable);
int sqg_timing_read(sqg_plan* plan, double* ms, int64_t* count, int32_t nkinds);

/* Host copies of the float64 wavenumbers and of the per-row dealias / drag
 * limits on |m_y| (for host-side checks of the masks; no GPU needed). */
int sqg_plan_host_tables(const sqg_plan* plan, double* k1d, int32_t* dmax, int32_t* dragmax);

const char* sqg_last_error_string(void);
int sqg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SQG_H */
