/*
 * n4b200 - N4 bias-field correction for NVIDIA B200 (sm_100a).
 *
 * C ABI.  Plain pointers and sizes only; every call returns an n4_status_t
 * and never exits or traps.  Volumes are float32, row-major [fx][fy][fz]
 * with fz fastest, exactly the layout of the reference N4 (cudaN4.cu:476).
 * A mask voxel is foreground when it is non-zero: float masks as in the
 * reference, or byte masks (uint8_t, with N4_FLAG_MASK_U8).
 *
 * Device-pointer calls are asynchronous on the given stream (NULL = the
 * legacy default stream) unless a report is requested; host-pointer calls
 * are synchronous.  One context per host thread; a context owns every
 * workspace, so no call allocates inside the iteration loop.
 */
#ifndef N4B200_H
#define N4B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define N4_MAX_LEVELS 8

typedef enum {
  N4_OK = 0,
  N4_ERR_INVALID_ARG = 1,
  N4_ERR_UNSUPPORTED_SPLINE_ORDER = 2,
  N4_ERR_EMPTY_MASK = 3,
  N4_ERR_OOM = 4,
  N4_ERR_CUDA = 5,
  N4_ERR_TIMEOUT = 6,        /* a bounded device-side wait gave up */
  N4_ERR_NONFINITE = 7,      /* non-finite intensity inside the mask */
  N4_ERR_TOO_LARGE = 8,      /* request exceeds a documented limit */
  N4_ERR_NO_DEVICE = 9
} n4_status_t;

/* Flags (n4_params_t.flags).  Defaults follow N4.py. */
#define N4_FLAG_CV_DDOF1        0x1u  /* CV standard deviation over N-1 (cudaN4.cu:979)          */
#define N4_FLAG_FIT_ZERO_DEN    0x2u  /* lattice = den != 0 ? num/den : 0 (cudaN4.cu:123-127)     */
#define N4_FLAG_INPLACE_THRESH  0x4u  /* write im = mask = 0 where im <= low_value back into the   */
                                      /* caller's buffers, as the reference does (cudaN4.cu:1459) */
#define N4_FLAG_FORCE_GRID      0x8u  /* run the whole-GPU path even when a cluster path fits      */
#define N4_FLAG_FORCE_CLUSTER   0x10u /* fail with N4_ERR_TOO_LARGE rather than use the grid path */
/* Bits 8-12: run the cluster path with exactly k CTAs per volume (1..16),
 * overriding the autotuner; N4_ERR_TOO_LARGE when a volume's share does not
 * fit one CTA's shared memory.  0 = choose automatically. */
#define N4_FLAG_CLUSTER_SIZE(k) (((unsigned int)(k) & 31u) << 8)
/* Bit 13: 512 threads per CTA instead of 1024 (twice the registers per
 * thread); overrides the autotuner's choice of threads. */
#define N4_FLAG_CTA_512         0x2000u
/* Bit 14: every mask pointer of a run (n4_run, n4_run_host, n4_run_batched*,
 * n4_batch_graph_create*, n4_warm_inputs, n4_autotune) points to uint8_t
 * bytes, one per voxel, non-zero = foreground, instead of floats (a quarter of
 * the bytes to move; the component entry points take float masks). */
#define N4_FLAG_MASK_U8         0x4000u
/* Bits 16-18: a batch on the cluster path runs as k sub-batches, each
 * sub-batch's prologue, warm start and correction overlapping the other
 * sub-batches' N4 iterations on the SMs the clusters leave free (1 = one
 * pass, no overlap; 0 = choose: one sub-batch per two waves of clusters, at
 * most 4).  Every volume's result is the same either way. */
#define N4_FLAG_SUB_BATCHES(k)  (((unsigned int)(k) & 7u) << 16)
/* Bits 19-23: with two or more sub-batches, each sub-batch runs on the
 * smallest cluster size >= k (of 2, 4, 6, 8, 12, 16) that holds its volumes
 * instead of one size for the whole batch.  Volumes are planned largest
 * first, so later sub-batches take smaller clusters, more of them side by
 * side.  0 = one cluster size (or the autotuner's record).  A volume's result
 * is its single run's on the same cluster size. */
#define N4_FLAG_SUB_CLUSTER_FLOOR(k) (((unsigned int)(k) & 31u) << 19)

/* Mirrors N4Param (cudaN4.h:24-94).  Obtain defaults from n4_params_default. */
typedef struct {
  unsigned int NumberOfHistogramBins;            /* 200                                */
  float WienerFilterNoise;                       /* 0.01                               */
  float BiasFieldFullWidthAtHalfMaximum;         /* 0.15                               */
  unsigned int NumberOfControlPoints_x;          /* 4 (first level)                    */
  unsigned int NumberOfControlPoints_y;          /* 4                                  */
  unsigned int NumberOfControlPoints_z;          /* 4                                  */
  unsigned int NumberOfFittingLevels;            /* 4                                  */
  unsigned int MaximumNumberOfIterations[N4_MAX_LEVELS]; /* 50 at every level          */
  float ConvergenceThreshold;                    /* 0.001                              */
  float low_value;                               /* 10 (reference default)             */
  unsigned int ShrinkFactor;                     /* 1 (not in the reference)           */
  unsigned int SplineOrder;                      /* 3; no other order is supported     */
  float FitEpsilon;                              /* 1e-3: num/(den+eps) as in N4.py    */
  unsigned int flags;                            /* N4_FLAG_*                          */
} n4_params_t;

/* Per-volume outcome. */
typedef struct {
  int status;                                    /* n4_status_t                        */
  int levels;                                    /* levels run                         */
  int iterations[N4_MAX_LEVELS];                 /* iterations run per level           */
  float final_cv[N4_MAX_LEVELS];                 /* last convergence value per level   */
  int warm_start_used;                           /* 1 if the warm lattice was kept     */
  float first_cv_warm, first_cv_plain;           /* first-iteration CVs (warm start)   */
  long long foreground;                          /* masked voxels at fitting resolution*/
  int path;                                      /* 1 = cluster, 2 = whole-GPU grid    */
  int cluster_size;                              /* CTAs per volume                    */
  unsigned long long device_begin_ns;            /* GPU global timer when the volume's */
  unsigned long long device_end_ns;              /*   levels began / ended (ns)        */
  int sm;                                        /* SM of the CTA that led the volume  */
  int reserved;
} n4_report_t;

/* One volume of a batch (device pointers). */
typedef struct {
  const float *im;            /* [fx][fy][fz]                                    */
  const float *mask;          /* float mask or NULL (NULL = every voxel)         */
  unsigned int fx, fy, fz;
  float *im_normalized;       /* [fx][fy][fz] output                             */
  float *lattice;             /* final lattice, n4_lattice_size() floats         */
  float *bias_field;          /* optional exp(log bias) output, may be NULL      */
  const float *warm_lattice;  /* optional first-level lattice, may be NULL       */
} n4_volume_t;

typedef struct n4_context n4_context_t;
typedef struct n4_encoder n4_encoder_t;   /* the learned warm start, see below */

/* Defaults of N4Param (cudaN4.h:24-94). */
void n4_params_default(n4_params_t *p);

/* Number of control points per axis at the last level and their product
 * (cudaN4.h:359, main.cpp:87-92). */
n4_status_t n4_lattice_dims(const n4_params_t *p, unsigned int dims[3], size_t *count);

/* No counterpart in the reference (it has no shrink factor).  Checks a
 * volume of fx*fy*fz voxels against the parameters exactly as n4_run does
 * before it touches the GPU (shrink divisibility, size limits) and returns
 * the fitting-grid dimensions (fx, fy, fz) / ShrinkFactor.  Needs no GPU. */
n4_status_t n4_fitting_dims(const n4_params_t *p, unsigned int fx, unsigned int fy, unsigned int fz,
                            unsigned int dims[3]);

const char *n4_status_string(int status);
/* Message of the last failed call on this thread. */
const char *n4_last_error_string(void);
const char *n4_version(void);

n4_status_t n4_create(n4_context_t **ctx, int device);
n4_status_t n4_destroy(n4_context_t *ctx);

/*
 * Whole N4 on one volume, device pointers.  Replaces
 *   void N4(float *d_im, float *d_mask, unsigned fx, fy, fz, N4Param&, N4Data&,
 *           float *d_im_normalized, float *d_lattice, float *d_biasField)
 * (cudaN4.h:343-365).  Inputs are not modified unless N4_FLAG_INPLACE_THRESH.
 * `stream` is a cudaStream_t.  With `report` non-NULL the call waits for the
 * result and returns the volume's status; with NULL it only enqueues.
 */
n4_status_t n4_run(n4_context_t *ctx, const n4_params_t *p,
                   const float *d_im, const float *d_mask,
                   unsigned int fx, unsigned int fy, unsigned int fz,
                   float *d_im_normalized, float *d_lattice, float *d_bias_field,
                   const float *d_warm_lattice, void *stream, n4_report_t *report);

/* Host-pointer twin; replaces testN4 (cudaN4.h:367-387).  Synchronous. */
n4_status_t n4_run_host(n4_context_t *ctx, const n4_params_t *p,
                        const float *h_im, const float *h_mask,
                        unsigned int fx, unsigned int fy, unsigned int fz,
                        float *h_im_normalized, float *h_lattice, float *h_bias_field,
                        const float *h_warm_lattice, n4_report_t *report);

/* Batched host-pointer twin (testN4, cudaN4.h:367-387, corrects one volume
 * per call).  vols[i] holds HOST pointers (im, mask, outputs, optional bias
 * and warm lattice).  The volumes are corrected in sub-batches of `per`
 * (0: the library's choice, 8) on four lanes: a lane's stream carries its
 * sub-batch's uploads into the lane's device staging slot, the batched run
 * and the downloads, the runs of successive sub-batches follow one another
 * (one context), and the copies of the other lanes overlap them, so the host
 * link and the GPU stay busy together.  Host buffers should be page-locked
 * (cudaHostAlloc / cudaHostRegister) for the copies to overlap.  enc: the
 * learned warm start (as n4_run_batched_warm) or NULL.  reports: n entries
 * or NULL.  device_ms (may be NULL): GPU time from the first upload to the
 * last download.  Synchronous. */
n4_status_t n4_run_batched_host(n4_context_t *ctx, const n4_params_t *p, int n,
                                const n4_volume_t *vols, int per, n4_encoder_t *enc,
                                n4_report_t *reports, float *device_ms);

/* Many volumes of uneven sizes in one persistent launch (no counterpart in
 * the reference, which corrects one volume per call).  `reports` (n entries)
 * may be NULL for a fully asynchronous call. */
n4_status_t n4_run_batched(n4_context_t *ctx, const n4_params_t *p, int n,
                           const n4_volume_t *vols, void *stream, n4_report_t *reports);

/* Wait for the context's last asynchronous run and fill its reports. */
n4_status_t n4_sync(n4_context_t *ctx, n4_report_t *reports, int n);

/* A batched run recorded once as a CUDA graph (no counterpart in the
 * reference).  Every launch repeats the run on the same buffers (the
 * caller may refill the inputs in between) without host-side planning.
 * The graph uses the context's workspaces as sized at its creation: do not
 * run other work on the context while a launch is in flight, and give each
 * graph a context of its own (a later run that needs larger workspaces
 * reallocates them under the graph). */
typedef struct n4_batch_graph n4_batch_graph_t;
n4_status_t n4_batch_graph_create(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols,
                                  n4_batch_graph_t **graph);
n4_status_t n4_batch_graph_launch(n4_batch_graph_t *graph, void *stream);
/* Wait for the last launch and fill its reports (n entries, may be NULL). */
n4_status_t n4_batch_graph_sync(n4_batch_graph_t *graph, n4_report_t *reports, int n);
n4_status_t n4_batch_graph_destroy(n4_batch_graph_t *graph);
/* The recorded run's kernel launches per graph launch (the library's own
 * kernels) and its sub-batches (N4_FLAG_SUB_BATCHES); either may be NULL. */
n4_status_t n4_batch_graph_info(const n4_batch_graph_t *graph, int *kernel_launches, int *sub_batches);

/* ---- autotuning (no counterpart in the reference) ----
 * n4_autotune runs the given volumes once per execution configuration that
 * fits them: thread-block clusters of 16, 12, 8, 6, 4 and 2 CTAs per volume
 * (a cluster keeps its volume in shared memory; smaller clusters run more
 * volumes side by side) and, for a single volume, the whole-GPU path, each
 * with 1024, 768 and 512 threads per CTA; then, on the fastest, every tile
 * shape of the full-resolution correction (rows per tile x threads per CTA,
 * timed by the correction stage's own device time) and 1 to 4 overlapped
 * sub-batches (N4_FLAG_SUB_BATCHES).  It records all three in the
 * context under the key (lattice, levels, bins, shrink factor, fitting-grid
 * size of every volume, in order; with the shrink factor that fixes the
 * full-resolution sizes); later n4_run, n4_run_batched and
 * n4_batch_graph_create calls with the same key use them unless a FORCE flag
 * is set.  The reference's tiles are fixed (6x6x6 span blocks,
 * cudaN4.cu:1190-1215, 1300-1330).  The outputs of the volumes are written as
 * by a run.  Synchronous. */
#define N4_TUNE_MAX 24
typedef struct {
  int candidates;                  /* configurations timed                   */
  int cluster_size[N4_TUNE_MAX];   /* CTAs per volume; 0 = whole-GPU path    */
  int threads[N4_TUNE_MAX];        /* threads per CTA                        */
  float ms[N4_TUNE_MAX];           /* device time of one run of the volumes  */
  int chosen;                      /* index of the configuration recorded    */
  /* tile shapes of the full-resolution correction on the chosen path */
  int corr_candidates;
  int corr_rows[N4_TUNE_MAX];      /* full-resolution rows per tile          */
  int corr_threads[N4_TUNE_MAX];   /* threads per CTA                        */
  float corr_ms[N4_TUNE_MAX];      /* device time of the correction stage    */
  int corr_chosen;
  /* overlapped sub-batches on the chosen path and tile (cluster path, two
   * or more volumes; 0 candidates otherwise): 1..4 of equal size, then 3
   * and 4 with the first and last half the size of the others, all on the
   * chosen cluster size; then per-sub-batch cluster sizes (sub_adapt > 0:
   * each sub-batch on the smallest size >= sub_adapt that holds its
   * volumes; the volumes are planned largest first, so later sub-batches
   * take smaller clusters), on the best split and on 4 tapered, for each
   * floor that gives sizes not timed before */
  int sub_candidates;
  int sub_count[N4_TUNE_MAX];      /* sub-batches                            */
  int sub_tapered[N4_TUNE_MAX];    /* 1: half-size first and last            */
  float sub_ms[N4_TUNE_MAX];       /* device time of one run                 */
  int sub_chosen;                  /* index of the candidate recorded        */
  int sub_adapt[N4_TUNE_MAX];      /* 0: one cluster size; > 0: the floor    */
} n4_tune_report_t;

n4_status_t n4_autotune(n4_context_t *ctx, const n4_params_t *params, int n,
                        const n4_volume_t *volumes, void *stream, n4_tune_report_t *report);

/* ---- measurement (no counterpart in the reference) ----
 * With profiling enabled, every call records CUDA events around its kernels
 * on its stream; n4_last_timings waits for the last profiled call and
 * returns the device time of its stages:
 *   n4_run / n4_run_batched: [0] threshold/shrink/log, [1] all levels and
 *     iterations, [2] full-resolution tables, [3] evaluation + im / exp(b);
 *   n4_fit_bspline3d: [0] z contraction (one pass over field and mask),
 *     [1] y contraction, [2] x contraction and division, [3] 0;
 *   n4_evaluate_bspline3d: [0] tables, [1] dense evaluation, [2], [3] 0. */
typedef struct {
  float stage_ms[4];
  int launches;            /* kernels launched by the call                */
  long long fit_voxels;    /* fitting-grid voxels of the call             */
  long long full_voxels;   /* full-resolution voxels of the call          */
  int fit_rows, fit_step;  /* z-contraction shape of a fit call (-1: none) */
  int fit_depth, reserved;
  int correct_rows, correct_threads;   /* correction tile (-1: none)      */
} n4_timings_t;

n4_status_t n4_set_profiling(n4_context_t *ctx, int enable);
n4_status_t n4_last_timings(n4_context_t *ctx, n4_timings_t *t);

/* ---- components (unit-level parity with the reference's entry points) ---- */

/* Replaces FitBspline3D (cudaN4.h:313-325): lattice[ncpt] fitted to `field`
 * over the voxels where mask != 0.  eps as n4_params_t.FitEpsilon;
 * zero_den selects N4_FLAG_FIT_ZERO_DEN semantics. */
n4_status_t n4_fit_bspline3d(n4_context_t *ctx, const float *d_field, const float *d_mask,
                             unsigned int ncpt_x, unsigned int ncpt_y, unsigned int ncpt_z,
                             unsigned int fx, unsigned int fy, unsigned int fz,
                             float eps, int zero_den, float *d_lattice, void *stream);

/* No counterpart in the reference (its FitBspline3D cudaMallocs and frees
 * three buffers per call, cudaN4.cu:1275-1365).  The same fit as
 * n4_fit_bspline3d for callers that must not allocate device memory during
 * the call, e.g. code running under a fixed memory budget or a caching
 * allocator that owns the whole device: it takes no context and makes no
 * cudaMalloc/cudaFree or allocating library call.  Its scratch is one fixed
 * 8 MiB device array per device, which holds the axis tables plus
 * fx*fy*ncpt_z*8 + fx*ncpt_y*ncpt_z*8 bytes (e.g. 256x256 rows with up to
 * 15 control points along z); larger fits return N4_ERR_TOO_LARGE and need
 * n4_fit_bspline3d.  The first call on a device (and again the first one in
 * a context made after cudaDeviceReset) looks up the array's address; make
 * it before any stream capture.  That first call may also be the one that
 * loads the library's device code (lazy module loading), which is when the
 * 8 MiB are reserved; later calls reserve nothing.  Calls on one device share the
 * scratch: two calls that may overlap in time (different streams or host
 * threads) race and must be ordered by the caller.  Runs on the current
 * device, asynchronously on `stream`. */
n4_status_t n4_fit_bspline3d_noalloc(const float *d_field, const float *d_mask,
                                     unsigned int ncpt_x, unsigned int ncpt_y, unsigned int ncpt_z,
                                     unsigned int fx, unsigned int fy, unsigned int fz,
                                     float eps, int zero_den, float *d_lattice, void *stream);

/* No counterpart in the reference (its fit and evaluation tiles are fixed:
 * 6x6x6 span blocks, cudaN4.cu:1190-1215, 1300-1330).  Times every shape of
 * n4_fit_bspline3d's z contraction that the field's alignment allows
 * (voxels per load step, steps in flight, rows per CTA) and every tile shape
 * of n4_evaluate_bspline3d (rows per tile, threads per CTA) on an fx*fy*fz
 * field with an ncpt lattice, each launch after L2 has been evicted, and
 * records the fastest of each in the context under (fx, fy, fz, ncpt and,
 * for the fit, the alignment class of field and mask): later calls of those
 * two entry points with that key use them.  d_field/d_mask: a field to fit;
 * d_lattice: ncpt floats, receives the fit; d_out: fx*fy*fz floats, written
 * by the evaluation candidates.  Synchronous. */
typedef struct {
  int fit_candidates;
  int fit_step[N4_TUNE_MAX];       /* voxels per load step (0: staged kernel) */
  int fit_depth[N4_TUNE_MAX];      /* load steps in flight per thread         */
  int fit_rows[N4_TUNE_MAX];       /* field rows per CTA                      */
  float fit_ms[N4_TUNE_MAX];       /* z contraction, L2 evicted               */
  int fit_chosen, fit_shape;       /* candidate index, library shape index    */
  int eval_candidates;
  int eval_rows[N4_TUNE_MAX];      /* field rows per tile                     */
  int eval_threads[N4_TUNE_MAX];   /* threads per CTA                         */
  float eval_ms[N4_TUNE_MAX];      /* dense evaluation, L2 evicted            */
  int eval_chosen, eval_shape;
} n4_component_tune_t;
n4_status_t n4_autotune_components(n4_context_t *ctx, const float *d_field, const float *d_mask,
                                   unsigned int ncpt_x, unsigned int ncpt_y, unsigned int ncpt_z,
                                   unsigned int fx, unsigned int fy, unsigned int fz,
                                   float *d_lattice, float *d_out, void *stream,
                                   n4_component_tune_t *report);

/* Replaces EvaluateBspline3D (cudaN4.h:288-298). */
n4_status_t n4_evaluate_bspline3d(n4_context_t *ctx, const float *d_lattice,
                                  unsigned int ncpt_x, unsigned int ncpt_y, unsigned int ncpt_z,
                                  unsigned int fx, unsigned int fy, unsigned int fz,
                                  float *d_fitted, void *stream);

/* Replaces upsampleLattice3D_gpu (cudaN4.h:269-276): (n+3) -> (2n+3) per axis. */
n4_status_t n4_upsample_lattice3d(n4_context_t *ctx, const float *d_lattice,
                                  unsigned int ncpt_x, unsigned int ncpt_y, unsigned int ncpt_z,
                                  float *d_lattice_upsample, void *stream);

/* Replaces sharpenImage (cudaN4.h:198-234): histogram sharpening of the log
 * image over the mask; masked-out voxels of the output are 0.  Optional
 * outputs: bin range and the n_bins-entry intensity map E.  Synchronous. */
n4_status_t n4_sharpen_image(n4_context_t *ctx, const float *d_before, const float *d_mask,
                             unsigned int n, unsigned int bins, float wiener, float fwhm,
                             float *d_after, float *bin_min, float *bin_max, float *h_E);

/* Replaces calculateConvergenceMeasurement (cudaN4.h:249-257): std/mean of
 * exp(field1 - field2) over the mask, ddof 0 (N4.py) or 1 (cudaN4).
 * Synchronous; the result is returned, not written into the threshold. */
n4_status_t n4_convergence(n4_context_t *ctx, const float *d_field1, const float *d_field2,
                           const float *d_mask, unsigned int n, int ddof, double *cv);

/* ---- learned warm start (no counterpart in the reference) ----
 * A small 3-D convolutional encoder (4 conv 3x3x3 stride 2 layers of
 * 16/32/64/64 channels with ReLU, then a linear layer to 64 outputs) that
 * predicts the first-level 4x4x4 log-bias lattice from the masked log
 * fitting grid average-pooled to 32x32x24.  BF16 weights and activations,
 * FP32 accumulation on the tensor cores; FP32 master weights and Adam
 * moments.  Inputs are device arrays of batch x 32 x 32 x 24 BF16 values
 * (n4_warm_inputs writes them); outputs batch x 64 floats, first-level
 * lattices (n4_run_batched_warm uses them as warm starts). */

size_t n4_encoder_num_params(void);
n4_status_t n4_encoder_create(n4_encoder_t **enc, int device, int max_batch);
n4_status_t n4_encoder_destroy(n4_encoder_t *enc);
/* Host FP32 parameter vector (n4_encoder_num_params entries); resets Adam. */
n4_status_t n4_encoder_set_params(n4_encoder_t *enc, const float *h_params, size_t n);
/* Parameters and the gradients of the last train step (either may be NULL). */
n4_status_t n4_encoder_get_params(n4_encoder_t *enc, float *h_params, float *h_grads, size_t n);
n4_status_t n4_encoder_predict(n4_encoder_t *enc, const void *d_x, int batch, float *d_out, void *stream);
/* Forward, MSE against d_target (batch x 64), backward; an Adam step when
 * lr > 0.  h_loss (may be NULL) receives the batch loss (synchronises). */
n4_status_t n4_encoder_train_step(n4_encoder_t *enc, const void *d_x, const float *d_target, int batch,
                                  float lr, float *h_loss, void *stream);


/* ---- learned warm start inside a batched run (no counterpart in the
 * reference) ----
 * The network input of a volume is its masked log fitting grid (the
 * threshold/shrink/log prologue of a run, background excluded) averaged over
 * 32x32x24 adaptive cells, BF16 [32][32][24].  n4_warm_inputs writes the
 * inputs of n volumes to d_x (n x 24576 BF16 values) without running N4
 * (training data).  n4_run_batched_warm runs prologue -> pooling -> encoder
 * -> N4 with the predicted lattices as warm starts -> correction on the
 * stream, with the usual first-iteration rule per volume (a prediction whose
 * first convergence value exceeds the zero lattice's is discarded); the
 * volumes' warm_lattice fields must be NULL and the first-level lattice
 * 4x4x4.  n4_batch_graph_create_warm records the same run as a CUDA graph.
 * The encoder's buffers are used by one run at a time. */
n4_status_t n4_warm_inputs(n4_context_t *ctx, const n4_params_t *p, int n,
                           const n4_volume_t *vols, void *d_x, void *stream);
n4_status_t n4_run_batched_warm(n4_context_t *ctx, const n4_params_t *p, int n,
                                const n4_volume_t *vols, n4_encoder_t *encoder, void *stream,
                                n4_report_t *reports);
n4_status_t n4_batch_graph_create_warm(n4_context_t *ctx, const n4_params_t *p, int n,
                                       const n4_volume_t *vols, n4_encoder_t *encoder,
                                       n4_batch_graph_t **graph);

#ifdef __cplusplus
}
#endif
#endif /* N4B200_H */
