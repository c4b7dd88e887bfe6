/*
 * ppf.h -- C ABI of libppf.so, the B200 (sm_100a) particle-filter library.
 *
 * The library replaces the per-observation loop of pypomp's particle filter
 * (the jitted XLA programs behind pypomp's functional API) for the built-in
 * models LG, SV and Ricker.  Each entry point is the drop-in for one reference
 * function; the Python host layer (pypomp_b200.functional) binds them with
 * ctypes exactly as a maintainer would bind them from pypomp.
 *
 * Conventions
 *  - Every pointer argument is DEVICE memory owned by the caller, unless the
 *    comment says host.  The library allocates nothing on the device: all
 *    scratch lives in the caller's workspace (size from *_workspace_bytes).
 *  - Calls are asynchronous on the given stream and reentrant across distinct
 *    (stream, workspace) pairs.
 *  - Return codes: PPF_OK, PPF_EINVAL (bad sizes / null pointers / J < 1),
 *    PPF_ECUDA (launch or runtime error), PPF_ETIMEOUT (a bounded device-side
 *    wait gave up; results are invalid), PPF_EUNSUPPORTED, PPF_EINTERNAL (a
 *    device-side consistency check failed and the access was skipped).
 *  - Arithmetic (the exact definitions every path and the C oracle share):
 *      state and log-weights float32, model math in a fixed operation order
 *      with the elementary functions of ppf_detmath.h;
 *      e_j = exp(w_j - max w) rounded to the fixed-point integer
 *      q_j = rint(e_j * 2^40) (uint64), CDF C_j = q_0 + ... + q_j exact;
 *      systematic points with u32 = floor(U * 2^32):
 *      parent(k) = #{ j : C_j * J * 2^32 <= (u32 + k 2^32) * C_{J-1} }
 *      (128-bit exact; this is searchsorted(cdf, (U+k)/J, side="right"));
 *      log-likelihood terms and their running sum in float64.
 *    J is limited to 2^21 so that the fixed-point total fits 62 bits.
 */
#ifndef PPF_H
#define PPF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPF_OK 0
#define PPF_EINVAL 1
#define PPF_ECUDA 2
#define PPF_ETIMEOUT 3
#define PPF_EUNSUPPORTED 4
#define PPF_EINTERNAL 5
#define PPF_ESCRATCH 6

#define PPF_MAX_J (1 << 21)

/* Built-in models (pypomp/models/linear_gaussian.py:337 LG; the SV and Ricker
 * factories follow the same pattern, pypomp/models/spx.py:161). */
enum { PPF_MODEL_LG = 1, PPF_MODEL_SV = 2, PPF_MODEL_RICKER = 3 };

typedef struct ppf_model {
  int32_t kind;     /* PPF_MODEL_* */
  int32_t dx;       /* state dimension (LG 1..9, SV 2, Ricker 1) */
  int32_t dy;       /* observation dimension (LG 1..9, SV 1, Ricker 1) */
  int32_t n_params; /* P, the canonical parameter count */
  float dt;         /* SV time step (1/252); ignored by the other models */
  int32_t reserved;
} ppf_model;

/* Flags */
#define PPF_F_CLL (1u << 0)      /* per-step conditional log-likelihood */
#define PPF_F_ESS (1u << 1)      /* per-step effective sample size */
#define PPF_F_FMEAN (1u << 2)    /* per-step filter mean */
#define PPF_F_PMEAN (1u << 3)    /* per-step prediction mean */
#define PPF_F_INJECT (1u << 4)   /* read noise from inj_* instead of Philox */
#define PPF_F_SAVE_ANC (1u << 5) /* write resampling ancestors */
#define PPF_F_SAVE_W (1u << 6)   /* write unnormalised log-weights */
#define PPF_F_EST (1u << 7)      /* theta on the estimation scale */
/* ppf_mop / ppf_perfilter: parameters on the natural scale (an identity
 * parameter transform, pypomp's ParTrans(); the default for these two entry
 * points is the estimation scale) */
#define PPF_F_NATURAL (1u << 8)
/* ppf_pfilter (stream and resident paths), ppf_mop, ppf_perfilter: capture
 * the call's launch sequence into a CUDA graph on first use and replay the
 * graph on later calls whose descriptor is byte-identical (same buffers, same
 * shapes, same flags).  The caller keeps those buffers alive and unchanged in
 * layout while it reuses the descriptor; a call made while the stream is
 * already being captured launches directly into that capture.  Host-side
 * cache of 16 graphs per process, not thread-safe. */
#define PPF_F_GRAPH (1u << 9)
/* ppf_perfilter: use the streaming kernels even where the cluster-resident
 * path would be chosen (small swarms); for comparisons and tests */
#define PPF_F_NO_CLUSTER (1u << 10)
/* ppf_mop / ppf_mop_backward: use one launch per step even where the
 * persistent form (the forward in one cooperative launch, the adjoint sweep in
 * another, grid barriers between the steps) would be chosen; for comparisons
 * and tests.  Both forms give the same forward results bit for bit. */
#define PPF_F_NO_PERSIST (1u << 11)
/* ppf_pfilter, streaming path, Philox draws: the hardware approximations of
 * the special-function units for the Box-Muller transform (log, sqrt, sin,
 * cos) and for the resampling weights' exponential, and fused multiply-adds
 * in the model arithmetic.  The fixed-point resampling CDF, the Philox
 * counters and the float64 log-likelihood sums are unchanged.  Results are
 * statistically equivalent to the exact arithmetic (log-weights of the same
 * particles agree to ~1e-6 relative) but not bit-identical with the C oracle.
 * Ignored with PPF_F_INJECT and on the other paths. */
#define PPF_F_FAST (1u << 12)
/* ppf_mop / ppf_mop_backward: the DPOP objective instead of MOP-alpha
 * (pypomp/core/algorithms/dpop.py:34-243).  State component
 * process_weight_index of the predicted particles holds the transition
 * log-weight accumulated over the interval, and enters the carried weights
 * as pw - stop_gradient(pw) (dpop.py:203-209).  Its value is zero, so the
 * objective's value is MOP-alpha's; the gradient gains the adjoint of the
 * carried weight times d pw / d theta along each lineage. */
#define PPF_F_DPOP (1u << 13)

/* Execution paths; all produce bit-identical results. */
enum {
  PPF_PATH_AUTO = 0,     /* autotuner / size heuristic */
  PPF_PATH_PLAIN = 1,    /* one filter at a time, textbook kernels (1x baseline) */
  PPF_PATH_STREAM = 2,   /* batched, HBM-streaming, 2 fused kernels per step */
  PPF_PATH_RESIDENT = 3, /* batched, one CTA per filter, swarm in shared memory */
  PPF_PATH_CLUSTER = 4   /* one thread-block cluster (<= 16 CTAs) per filter, swarm in
                            the cluster's distributed shared memory for all T steps */
};

/* Inputs and outputs of one batched bootstrap particle filter call over F
 * filters.  Replaces _pfilter_internal / _pfilter_step
 * (pypomp/core/algorithms/pfilter.py:15-182) vmapped over parameter sets and
 * replicate keys (pfilter.py:185-207) and over panel units
 * (_chunked_panel_pfilter_internal, pfilter.py:248-304). */
typedef struct ppf_pfilter_desc {
  ppf_model model;
  int32_t J;            /* particles per filter, 1..PPF_MAX_J */
  int32_t F;            /* filters in the batch */
  int32_t T;            /* observations in the longest series */
  int32_t U;            /* number of observation series (panel units) */
  int32_t path;         /* PPF_PATH_* */
  uint32_t flags;       /* PPF_F_* */
  float thresh;         /* resampling threshold as in pfilter.py:159 */
  int32_t tile;         /* particles per CTA on the stream path: 2048, 512 or 256;
                           0 = the ppf_autotune choice for this shape, else the
                           largest tile that still launches 2 CTAs per SM */
  const float* theta;   /* [F][P] parameters (natural scale unless PPF_F_EST) */
  const float* ys;      /* [U][T][dy] observations */
  const float* ycon;    /* [U][T] per-observation constant (Ricker: lgamma(y+1)) or NULL */
  const int32_t* unit;  /* [F] series index of each filter, or NULL (series 0) */
  const int32_t* T_u;   /* [U] series lengths (ragged panels), or NULL (all T) */
  const uint64_t* seeds;/* [F] Philox keys */
  const float* inj_z0;  /* [F][J][n0] initial-state normals (PPF_F_INJECT) */
  const float* inj_z;   /* [F][T][J][nz] process normals (PPF_F_INJECT) */
  const float* inj_u;   /* [F][T] resampling uniforms in [0,1) (PPF_F_INJECT) */
  double* loglik;       /* out [F] log-likelihood estimate */
  double* cll;          /* out [F][T] (PPF_F_CLL) */
  float* ess;           /* out [F][T] (PPF_F_ESS) */
  float* fmean;         /* out [F][T][dx] (PPF_F_FMEAN) */
  float* pmean;         /* out [F][T][dx] (PPF_F_PMEAN) */
  int32_t* anc;         /* out [F][T][J] (PPF_F_SAVE_ANC) */
  float* logw;          /* out [F][T][J] (PPF_F_SAVE_W) */
  void* workspace;
  size_t ws_bytes;
} ppf_pfilter_desc;

/* MOP-alpha objective and gradient over F filters.  Replaces _mop_internal /
 * _mop_step (pypomp/core/algorithms/mop.py:19-135) vmapped over parameter
 * sets (mop.py:138) and its jax.value_and_grad (ad_helpers.py:32-54).
 * theta is on the ESTIMATION scale (the model's from_est is applied on the
 * device, mop.py:16).  value[f] = -sum_t ll_t (the negative MOP
 * log-likelihood); grad[f][p] = d value[f] / d theta[f][p] on the estimation
 * scale, from the adjoint sweep over stored ancestors with state checkpoints
 * every ckpt_every steps (0: ceil(sqrt(T))). */
typedef struct ppf_mop_desc {
  ppf_model model;
  int32_t J, F, T, U;
  uint32_t flags;         /* PPF_F_INJECT, PPF_F_NATURAL, PPF_F_GRAPH, PPF_F_DPOP */
  float alpha;            /* MOP discount in [0, 1] */
  int32_t ckpt_every;     /* 0 = ceil(sqrt(T)) */
  const float* theta;     /* [F][P] estimation scale */
  const float* ys;        /* [U][T][dy] */
  const float* ycon;      /* [U][T] or NULL */
  const int32_t* unit;    /* [F] or NULL */
  const int32_t* T_u;     /* [U] or NULL */
  const uint64_t* seeds;  /* [F] */
  const float* inj_z0;
  const float* inj_z;
  const float* inj_u;
  double* value;          /* out [F] */
  double* grad;           /* out [F][P] or NULL (value only) */
  int32_t* anc;           /* optional out [F][T][J] resampling ancestors */
  void* workspace;
  size_t ws_bytes;
  int32_t process_weight_index;   /* with PPF_F_DPOP: state component in [0, dx) */
} ppf_mop_desc;

size_t ppf_mop_workspace_bytes(const ppf_mop_desc* d);
int ppf_mop(const ppf_mop_desc* d, void* stream);

/* The adjoint sweep alone, for a caller that separates the forward from the
 * backward pass (a torch.autograd.Function; the reference gets both at once
 * from jax.value_and_grad at pypomp/core/algorithms/ad_helpers.py:6-54).
 * Call it after ppf_mop with the SAME descriptor and workspace, untouched in
 * between: the forward leaves the ancestors, first-child offsets, state
 * checkpoints and per-step maxima there.  Writes
 * grad[f][p] = dvalue[f] * d value[f] / d theta[f][p] (dvalue: device [F],
 * NULL for all ones); d->grad must be set. */
int ppf_mop_backward(const ppf_mop_desc* d, const double* dvalue, void* stream);

/* One IF2 iteration: the perturbed particle filter over F independent
 * parameter swarms.  Replaces _perfilter_internal / _perfilter_scan_body
 * (pypomp/core/algorithms/mif.py:88-258) with _resampler_thetas
 * (pypomp/core/algorithms/helpers.py:103-141); Pomp.mif / functional mif
 * (pypomp/functional/mif.py:15, pypomp/core/estimation_mixin.py:274) call it
 * once per iteration.  Each particle carries a parameter vector on the
 * estimation scale: perturbed by rw_sig0[p] * cool0[u] * N(0,1) before the
 * initial state is drawn, by rw_sig[p] * cool[u][t] * N(0,1) before step t;
 * state and vector are resampled together; measurement log-densities that
 * are NaN become log(1e-18) (mif.py:205-210).  Outputs: loglik[f] (sum of the
 * conditional log-likelihoods of the perturbed filter) and swarm_out, the
 * vectors after the last step's resampling.  The swarm layout is
 * parameter-major [F][P][J] (the reference holds (J, P) per replicate). */
typedef struct ppf_perfilter_desc {
  ppf_model model;
  int32_t J, F, T, U;
  uint32_t flags;          /* PPF_F_INJECT, PPF_F_CLL, PPF_F_SAVE_ANC, PPF_F_NATURAL */
  float thresh;            /* resample when max(nw) - min(nw) > log(thresh) */
  const float* swarm_in;   /* [F][P][J] estimation scale */
  float* swarm_out;        /* out [F][P][J]; may not alias swarm_in */
  const float* rw_sig;     /* [P] per-step random-walk sds (estimation scale) */
  const float* rw_sig0;    /* [P] sds of the t0-only perturbation */
  const float* cool;       /* [U][T] cooling factor of the step-t perturbation */
  const float* cool0;      /* [U] cooling factor of the t0 perturbation */
  const float* ys;         /* [U][T][dy] */
  const float* ycon;       /* [U][T] or NULL */
  const int32_t* unit;     /* [F] or NULL */
  const int32_t* T_u;      /* [U] or NULL */
  const uint64_t* seeds;   /* [F] */
  const float* inj_zp0;    /* [F][J][P] t0 perturbation normals (PPF_F_INJECT) */
  const float* inj_zp;     /* [F][T][J][P] per-step perturbation normals */
  const float* inj_z0;     /* [F][J][n_init] */
  const float* inj_z;      /* [F][T][J][n_step] */
  const float* inj_u;      /* [F][T] */
  double* loglik;          /* out [F] */
  double* cll;             /* out [F][T] (PPF_F_CLL) */
  int32_t* anc;            /* out [F][T][J] (PPF_F_SAVE_ANC) */
  void* workspace;
  size_t ws_bytes;
} ppf_perfilter_desc;

size_t ppf_perfilter_workspace_bytes(const ppf_perfilter_desc* d);
int ppf_perfilter(const ppf_perfilter_desc* d, void* stream);

/* Workspace bytes ppf_pfilter needs for this descriptor (pointers ignored). */
size_t ppf_pfilter_workspace_bytes(const ppf_pfilter_desc* d);

/* Run the batched particle filter.  `stream` is a cudaStream_t. */
int ppf_pfilter(const ppf_pfilter_desc* d, void* stream);

/* Measure the stream path's tile configurations (2048, 512, 256 particles
 * per CTA) on this descriptor -- a prefix of at most 16 observations, each
 * configuration run twice, timed with CUDA events on `stream` -- and remember
 * the fastest for descriptors of the same shape (model, J, F, U, injection)
 * that leave `tile` at 0.  Writes it to *best_tile (0 when the call would take
 * the resident path).  Runs the filter, so it overwrites the outputs and uses
 * the workspace; host-side cache, not thread-safe.  No counterpart in the
 * reference: XLA picks its own tiling. */
int ppf_autotune(const ppf_pfilter_desc* d, void* stream, int* best_tile);

/* Synchronise `stream` and report the device-side status of the last call
 * that used `workspace`: PPF_ETIMEOUT if a bounded wait gave up,
 * PPF_EINTERNAL if an index check failed, PPF_OK otherwise. */
int ppf_workspace_status(const void* workspace, void* stream);

/* Per-kernel timing of the calls made between begin and end: CUDA events are
 * recorded on the launch stream around each kernel (host-side bookkeeping
 * only).  ppf_profile_end synchronises and writes, for each kernel kind k < n,
 * the summed milliseconds ms[k] and launch count count[k].  Kinds: 0 init,
 * 1 weight-sum (tile totals and the filter's tile prefixes), 2 resample + propagate, 3 resident filter,
 * 4 plain-path step (four kernels), 5..8 MOP forward / recompute / adjoint /
 * IF2, 9 cluster filter, 10 simulation.  Not reentrant. */
int ppf_profile_begin(void);
int ppf_profile_end(double* ms, int* count, int n);

/* Test hook for the bounded device-side waits (the bulk-copy barrier waits of
 * the resampling kernel, the exchanges and grid barriers of the persistent
 * MOP kernels): set how many polls a wait makes before it gives up, for the calls
 * that follow (polls < 0 restores the default, 2^22; larger values are
 * clamped to it; 0 makes every such wait give up at its first check).  A wait
 * that gives up sets the workspace's error word, so ppf_workspace_status
 * reports PPF_ETIMEOUT and the call's outputs are invalid; a kernel whose
 * copy wait gave up still drains that copy before it continues.  CUDA graphs
 * cached by PPF_F_GRAPH keep the limit they were captured with.  Returns the
 * previous limit.  Host-side setting, not thread-safe.  No counterpart in the
 * reference (XLA has no device-side waits). */
long long ppf_debug_set_wait_limit(long long polls);

/* ppf_pfilter for callers that cannot allocate device memory.  No counterpart
 * in the reference: pypomp runs on JAX, whose runtime owns device memory.
 * Some callers of this library cannot hand it a workspace -- a host runtime
 * that owns the whole device pool and forbids other allocations, or plugin
 * code not allowed to call the CUDA allocator.  This entry point runs the same
 * filter as ppf_pfilter (descriptor fields `workspace` and `ws_bytes` are
 * ignored) on a scratch array of PPF_NOALLOC_SCRATCH_BYTES compiled into the
 * library, and allocates nothing.  A request whose workspace
 * (ppf_pfilter_workspace_bytes) exceeds that size returns PPF_ESCRATCH.  All
 * calls on a device share the array, so calls that overlap on the GPU race.
 * The first call on a device looks up the array's device address.  Every call
 * is synchronous: it waits for `stream` and then reads the device-side status,
 * so it returns PPF_EUNSUPPORTED, before doing any work, when `stream` is
 * being captured into a CUDA graph.  PPF_F_GRAPH is ignored (a cached graph
 * would need driver-side allocations); the launches go directly onto
 * `stream`. */
#define PPF_NOALLOC_SCRATCH_BYTES (16u << 20)
int ppf_pfilter_noalloc(const ppf_pfilter_desc* d, void* stream);

/* Simulated trajectories of the model: for each parameter set f and replicate
 * k, the initial state (rinit), then for each of the T observation times one
 * process step (rproc) and a draw of the observation (rmeas).  Replaces
 * _simulate_internal / _simulate_helper (pypomp/core/algorithms/simulate.py:15-142),
 * vmapped over parameter sets by functional.simulate
 * (pypomp/functional/simulate.py:8-72) and called by Pomp.simulate
 * (pypomp/core/estimation_mixin.py:1101-1222).  Output layouts are the
 * reference's: X[f][k][t][:] for t = 0..T (t = 0 the initial state) and
 * Y[f][k][t][:] for t = 0..T-1.  Replicate k of parameter set f draws from
 * the key seeds[f]: process normals as the filters' particle k does, the
 * observation's normals / counts from the measurement streams of
 * include/ppf_sample.h.  Ricker counts are Poisson draws (inversion below a
 * mean of 10, Hoermann's PTRS above). */
typedef struct ppf_simulate_desc {
  ppf_model model;
  int32_t F;               /* parameter sets, 1..65535 */
  int32_t nsim;            /* replicates per parameter set, >= 1 */
  int32_t T;               /* observation times, >= 0 */
  uint32_t flags;          /* PPF_F_EST: theta on the estimation scale */
  const float* theta;      /* [F][P] natural scale (estimation scale with PPF_F_EST) */
  const uint64_t* seeds;   /* [F] one key per parameter set */
  float* X;                /* out [F][nsim][T+1][dx] */
  float* Y;                /* out [F][nsim][T][dy] (may be NULL when T == 0) */
} ppf_simulate_desc;

int ppf_simulate(const ppf_simulate_desc* d, void* stream);

/* Human-readable message for a return code (static storage). */
const char* ppf_error_string(int code);

/* Library version string (static storage). */
const char* ppf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PPF_H */
