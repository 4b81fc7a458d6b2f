/*
 * sporco_b200 -- C ABI of the B200 (sm_100a) CBPDN ADMM solvers.
 *
 * Two layers of entry points:
 *
 * 1. Drop-in replacements for the reference's C ABI (same names, same
 *    argument meaning, same AlgOpt struct layout, host buffers in and out):
 *      cuda_wrapper_CBPDN      replaces sporco_cuda/src/cbpdn.h:10
 *      cuda_wrapper_CBPDN_GR   replaces sporco_cuda/src/cbpdn_grd.h:10-11
 *      clear_opts, default_opts, check_cuda_req
 *                              replace sporco_cuda/src/utils.h:18-20
 *      get_device_count, get_current_device, set_current_device,
 *      get_memory_info, get_device_name
 *                              replace the externs of sporco_cuda/util.pyx:3-7
 *                              (defined at sporco_cuda/src/utils.cu:146-176)
 *    The reference terminates the process on any CUDA error
 *    (error_check.cuh:10-21).  These return normally instead; the solver
 *    wrappers (void, as in the reference) record a status readable with
 *    sc_last_status() / sc_last_error(), and check_cuda_req returns -1.
 *
 * 2. The native interface (prefix sc_): device pointers, a caller-chosen
 *    CUDA stream, a caller-provided workspace, status codes, a batch of
 *    same-sized images per call, and the adjoint.  No allocation and no
 *    device-wide synchronisation happens inside sc_* solve calls, except the
 *    stream synchronisation needed to read the iteration count back.
 *
 * All arrays are C order.  Dictionaries are (M, Kr, Kc) float32, images
 * (H, W) float32, coefficient maps (M, H, W) float32 (the reference's internal
 * layout, cbpdn.pyx:97 / cbpdn.cu:136-149).
 */
#ifndef SPORCO_B200_H
#define SPORCO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Reference-compatible layer                                          */
/* ------------------------------------------------------------------ */

/* Same field order and types as AlgOpt (sporco_cuda/src/algopt.h:7-48). */
typedef struct AlgOpt {
  int MaxMainIter;
  float rho;
  float RhoRsdlRatio;
  float RhoScaling;
  float RhoRsdlTarget;
  float RelaxParam;
  float AbsStopTol;
  float RelStopTol;
  float *L1Weight;
  int L1_WEIGHT_M_SIZE;
  int L1_WEIGHT_ROW_SIZE;
  int L1_WEIGHT_COL_SIZE;
  int *Weight;
  int nWeight;
  int Verbose;
  int NonNegCoef;
  int NoBndryCross;
  int AuxVarObj;
  int HighMemSolve;
  int AutoRho;
  int AutoRhoScaling;
  int AutoRhoPeriod;
  int StdResiduals;
  int IMG_ROW_SIZE;
  int IMG_COL_SIZE;
  int DICT_M_SIZE;
  int DICT_ROW_SIZE;
  int DICT_COL_SIZE;
  float *GrdWeight;
  int WEIGHT_SIZE;
  int device;
} AlgOpt;

/* cbpdn.h:10.  D: host (M, Kr, Kc); S: host (H, W); Y: host (M, H, W). */
void cuda_wrapper_CBPDN(float *D, float *S, float lambda, void *opt, float *Y);
/* cbpdn_grd.h:10-11. */
void cuda_wrapper_CBPDN_GR(float *D, float *S, float lambda, float mu,
                           void *opt, float *Y);
/* utils.h:18-20 (clear_opts allocates nothing, unlike utils.cu:76-77). */
void clear_opts(void *opt);
void default_opts(void *opt);
int check_cuda_req(int device);
/* util.pyx:3-7 (return cudaError_t values as int). */
int get_device_count(void);
int get_current_device(int *dev);
int set_current_device(int dev);
int get_memory_info(size_t *free_bytes, size_t *total_bytes);
const char *get_device_name(int dev);

/* ------------------------------------------------------------------ */
/* Native layer                                                        */
/* ------------------------------------------------------------------ */

typedef enum sc_status {
  SC_OK = 0,
  SC_ERR_INVALID = 1,      /* bad sizes / arguments */
  SC_ERR_UNSUPPORTED = 2,  /* valid but beyond this build's limits */
  SC_ERR_WORKSPACE = 3,    /* workspace missing or too small */
  SC_ERR_CUDA = 4,         /* a CUDA runtime call failed */
  SC_ERR_NONFINITE = 5,    /* a residual became NaN or Inf */
  SC_ERR_OOM = 6,          /* device allocation failed */
  SC_ERR_CANCELLED = 7     /* the host set the cancel flag */
} sc_status;

/* Resolved solver options (every field set; see sc_options_from_algopt). */
typedef struct sc_options {
  int max_iter;         /* MaxMainIter */
  float relax;          /* RelaxParam */
  float abs_tol;        /* AbsStopTol */
  float rel_tol;        /* RelStopTol */
  int auto_rho;         /* AutoRho.Enabled */
  int auto_rho_period;  /* AutoRho.Period */
  float rho_scaling;    /* AutoRho.Scaling */
  float rsdl_ratio;     /* AutoRho.RsdlRatio */
  float rsdl_target;    /* AutoRho.RsdlTarget, <= 0: derive from lambda */
  int auto_scaling;     /* AutoRho.AutoScaling */
  int std_residuals;    /* AutoRho.StdResiduals */
  int record_itstat;    /* keep per-iteration statistics on the device (see sc_read_state) */
  int check_every;      /* host polls the stop flag every this many iterations (0: never) */
  int profile;          /* time every iteration kernel with CUDA events (sc_last_profile) */
  int nonneg;           /* NonNegCoef: project the coefficients onto >= 0 */
  int no_bndry_cross;   /* NoBndryCross: zero the last Kr - 1 rows and Kc - 1
                           columns of every map (filters crossing the bottom /
                           right boundary); neither touches the AMS map */
  int warm_start;       /* 0: start from Y = U = 0 (or U0) at rho0.  1: continue
                           the state an earlier solve of the same problem left
                           in this workspace (iterates, rho, iteration count;
                           max_iter more iterations), re-reading D and S (a
                           dictionary update between calls, as in dictionary
                           learning).  2: as 1, with D and S unchanged (their
                           spectra in the workspace are reused). */
} sc_options;

/* L1 weight layouts. */
enum { SC_L1_SCALAR = 0, SC_L1_PER_MAP = 1, SC_L1_FULL = 2 };

/* One batch of B images of equal size (H, W) sharing one dictionary.
 * Device pointers unless stated otherwise. */
typedef struct sc_problem {
  int B, H, W, M, Kr, Kc;
  const float *D;        /* (M, Kr, Kc) */
  const float *S;        /* (B, H, W) */
  const float *lmbda;    /* (B,) regularisation parameter per image */
  const float *rho0;     /* (B,) initial rho per image */
  int grd;               /* 1: gradient regularisation (cbpdngrd) */
  float mu;              /* gradient term weight */
  const float *wgrd;     /* (M,) GradWeight per map (grd only) */
  int l1_kind;           /* SC_L1_* */
  float l1_scalar;       /* SC_L1_SCALAR */
  const float *l1w;      /* (M,) or (M, H, W) */
  const int32_t *mask;   /* (B, H, W) AMS mask, map 0 is the impulse; NULL: none */
  float *Y;              /* (B, M, H, W) output; also the Y iterate */
  int wgrd_uniform;      /* grd only: 1 when all M GradWeight entries are equal */
  const float *U0;       /* (B, M, H, W) or NULL: start from Y (as given) and U0
                            instead of Y = U = 0 */
  float *U_out;          /* (B, M, H, W) or NULL: receives the final U */
} sc_problem;

typedef struct sc_result {
  int iterations;        /* largest iteration count of this call over the batch */
  double rho;            /* final rho of image 0 */
  double r, s;           /* final (normalised) residuals of image 0 */
} sc_result;

/* Workspace bytes for a problem (256-byte aligned pointer required). */
size_t sc_workspace_size(const sc_problem *p, const sc_options *o);

/* Fill sc_options from the reference's AlgOpt after default_opts. */
void sc_options_from_algopt(const AlgOpt *a, sc_options *o);

/* Solve; stream is a cudaStream_t (NULL: legacy default stream). */
int sc_cbpdn_solve(const sc_problem *p, const sc_options *o, void *workspace,
                   size_t workspace_bytes, sc_result *res, void *stream);

/* Several batches of different image sizes solved together (no reference
 * counterpart): problem i uses workspaces[i] (workspace_bytes[i]) and
 * streams[i] (NULL array: the legacy default stream for all).  Iterations of
 * all problems are launched in turn, each on its own stream, and every
 * problem stops on its own; res may be NULL or hold nprob results. */
int sc_cbpdn_solve_batch(const sc_problem *probs, int nprob, const sc_options *o,
                         void *const *workspaces, const size_t *workspace_bytes,
                         sc_result *res, void *const *streams);

/* Values per image and iteration in the statistics (sc_read_state). */
#define SC_ITSTAT_FIELDS 8

/* Per-image iteration counts (of the last solve call on this workspace) /
 * final rho / itstat after a solve, copied from the workspace of that solve
 * (host pointers; itstat may be NULL).  itstat is
 * (B, max_iter, 8) doubles per iteration: r, s, rho, eps_pri, eps_dua, then
 * the functional at Y, its data fidelity 0.5 ||sum_m d_m * y_m - s||^2 and
 * its L1 sum ||w y||_1 (the reference's Verbose columns, cbpdn.cu:438-517;
 * the functional adds lambda times the L1 sum and, with the gradient term,
 * mu/2 sum_m w_m ||grad y_m||^2; masked problems count the impulse map as a
 * filter, as the reference does).  Kept only with options.record_itstat. */
int sc_read_state(const sc_problem *p, const sc_options *o, const void *workspace,
                  int *iterations, double *rho, double *itstat, void *stream);

/* Forward 2-D real FFT of `count` (H, W) float32 arrays into half spectra
 * (count, H, W/2+1) complex64 (numpy rfft2 layout); test and tooling entry. */
int sc_rfft2(const float *x, void *xf, int count, int H, int W, void *stream);
/* Inverse of sc_rfft2 (numpy irfft2, normalised by 1/(H W)). */
int sc_irfft2(const void *xf, float *x, int count, int H, int W, void *stream);

/* sc_rfft2 without any device-memory allocation (no counterpart in the
 * reference).  For callers that must not allocate device memory -- code
 * running under a memory budget owned by another allocator, or
 * real-time callers that must not call into the allocator on their
 * critical path: its scratch (W + H twiddles) lives in a 64 KiB static
 * device array that every GPU loading this library holds until the process
 * exits.  Rejects H + W > 8192 with SC_ERR_UNSUPPORTED.  The first call on a
 * device looks up that array's device address and keeps it; make it before
 * any stream capture, and make no call on a device after cudaDeviceReset of
 * that device in the same process (the kept address belongs to the old
 * context).  All calls share the array, so calls that overlap on the GPU
 * race. */
int sc_rfft2_noalloc(const float *x, void *xf, int count, int H, int W, void *stream);

/* Per-kernel device time of the last solve run with options.profile set:
 * index 0 column pass, 1 row pass, 2 finalize, 3 rho fix-up. */
typedef struct sc_profile {
  double ms[4];
  int count[4];
} sc_profile;
int sc_last_profile(sc_profile *out);

/* Cancel every solve in progress in this process (any host thread): each
 * stops launching iterations at its next check (every options.check_every
 * iterations; without a stopping test it keeps at most two such chunks
 * queued), writes the iterates it reached and returns SC_ERR_CANCELLED.
 * Solves started after the call are not affected.  No counterpart in the
 * reference (which can only be stopped with its process). */
void sc_cancel(void);

/* Number of kernels this library has launched since it was loaded. */
unsigned long long sc_launch_count(void);

/* Differentiable unrolled cbpdn (no counterpart in the reference): exactly
 * o->max_iter = K plain-cbpdn ADMM iterations at the fixed rho p->rho0 (no
 * stopping test, no adaptive rho; p->grd = 0, p->mask = NULL, p->U0 = p->U_out
 * = NULL), and the reverse pass of those iterations.
 *   sc_unrolled_forward writes Y_K to p->Y and keeps the state V = Y + U
 *     every seg iterations in the workspace (seg: 1..K; ceil(sqrt(K)) balances memory
 *     against the one recomputation of each segment in the backward pass;
 *     seg = K with filters of at most 16 rows and compiled column lengths
 *     below 512 keeps the trace of every step instead, so that the backward
 *     recomputes nothing, in a workspace of about K (R + C) bytes).
 *   sc_unrolled_backward, after a forward call with the same problem,
 *     options, seg and workspace, takes gY = dLoss/dY_K (B, M, H, W) and
 *     writes dLoss/dD to gD (M, Kr, Kc) and dLoss/dS to gS (B, H, W).
 * The workspace (sc_unrolled_workspace_size bytes, 256-byte aligned) holds
 * the solver's own workspace, the checkpoints, one segment's V and x^ of
 * every step, and the gradient spectra.  Returns 0 when the problem is not
 * a plain fixed-rho cbpdn problem or seg is out of range. */
size_t sc_unrolled_workspace_size(const sc_problem *p, const sc_options *o, int seg);
int sc_unrolled_forward(const sc_problem *p, const sc_options *o, int seg, void *workspace,
                        size_t workspace_bytes, void *stream);
int sc_unrolled_backward(const sc_problem *p, const sc_options *o, int seg, void *workspace,
                         size_t workspace_bytes, const float *gY, float *gD, float *gS,
                         void *stream);

/* Last status / message recorded on the calling thread. */
int sc_last_status(void);
const char *sc_last_error(void);
const char *sc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SPORCO_B200_H */
