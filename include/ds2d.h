/*
 * ds2d.h -- C ABI of the B200-native DS2D time-stepping path.
 *
 * The reference exposes this path as the C++ class FD2DGPU_ELASTIC (FD2DGPU.cuh:124-422) plus
 * the per-shot driver ELSRTM_ROT_EXP_IMAGE_SINGLESHOT (FD2DGPU.cuh:429-430), called by
 * lsrtm_all_iteration (main.cpp:939-1035).  The entry points below replace that surface with a
 * plain C ABI: plain pointers and sizes, every call returns an int status (0 = DS2D_OK,
 * negative = DS2D_E_*), ds2d_last_error() gives the message.  Host arrays belong to the caller
 * and are copied in; the context owns all device memory.  One context per host thread.
 *
 * Array conventions follow the reference (idx = ix*nz + iz, z fastest):
 *   models / images   [allnx][allnz] float
 *   records           [ntr][nt] float per shot, shots concatenated in call order
 * Geometry is given in cells of the padded shot window: nxpml = nx + 2*pml, nzpml = allnz +
 * 2*pml, the window's first interior column sits at model column win_left.
 */
#ifndef DS2D_H
#define DS2D_H
#ifdef __cplusplus
extern "C" {
#endif

#define DS2D_OK 0
#define DS2D_E_ARG -1     /* invalid argument / geometry outside the model */
#define DS2D_E_CUDA -2    /* CUDA runtime error (message in ds2d_last_error) */
#define DS2D_E_NOMEM -3   /* device allocation failed */
#define DS2D_E_STATE -4   /* call order violated (e.g. models not set) */
#define DS2D_E_NUMERIC -5 /* non-finite value detected in a result */

enum { DS2D_BOUNDARY_PML = 0, DS2D_BOUNDARY_RANDOM = 1 };
enum { DS2D_STRIPS_F32 = 0, DS2D_STRIPS_F16 = 1, DS2D_STRIPS_BF16 = 2 };

typedef struct ds2d_ctx ds2d_ctx;

/* Grid of one run.  Replaces the constructor arguments of FD2DGPU_ELASTIC
 * (FD2DGPU.cu:1350-1352: dx, dz, dt, nxpml, nzpml, allnx, allnz, pml, nt; nop is fixed to 4 as
 * in main.cpp:1490). */
typedef struct {
  int allnx, allnz; /* full model */
  int nx;           /* largest shot window width in cells (the reference's single nx,
                       main.cpp:1421-1423); individual shots may be narrower (ds2d_shot.nx) */
  int pml;          /* PML width, or random-band width when boundary = RANDOM */
  int nt;           /* time steps */
  float dx, dz, dt;
} ds2d_grid;

typedef struct {
  int boundary;           /* DS2D_BOUNDARY_PML (strips saved) or _RANDOM (parameters line 9 rbc) */
  int strip_precision;    /* DS2D_STRIPS_*: storage of the saved boundary strips */
  int max_shots;          /* shots resident on the device at once (batch size) */
  int max_ntr;            /* upper bound of receivers per shot */
  unsigned long long seed;/* random-band seed */
  int device;             /* CUDA device ordinal */
} ds2d_opts;

/* One shot.  Replaces the public fields the reference sets before each driver call
 * (main.cpp:1019-1025: isx, isz, igz, delta_left + record_left_in_v) and the trace coordinates
 * of record_copytoGPU (FD2DGPU.cu:3537), already mapped to cells as
 * GPUrecord_scatterwavefield does (FD2DGPU.cu:3097: igx = pml + (gc - ngx_left)/dx). */
typedef struct {
  int win_left;   /* model column of the first interior column of the window */
  int isx, isz;   /* source cell (padded window coordinates) */
  int igz;        /* receiver row */
  int ntr;        /* receivers of this shot (<= max_ntr) */
  const int *igx; /* ntr distinct receiver columns (padded window coordinates) */
  int nx;         /* this shot's window width (0 = grid.nx, the maximum).  The reference
                     requires one width for all shots and proceeds with a wrong one otherwise
                     (main.cpp:1010-1017); here shots of a batch may differ. */
} ds2d_shot;

/* FD2DGPU_ELASTIC::FD2DGPU_ELASTIC (FD2DGPU.cu:1350). */
int ds2d_create(const ds2d_grid *grid, const ds2d_opts *opts, ds2d_ctx **out);
/* FD2DGPU_ELASTIC::~FD2DGPU_ELASTIC (FD2DGPU.cu:1640). */
int ds2d_destroy(ds2d_ctx *ctx);
const char *ds2d_last_error(const ds2d_ctx *ctx);

/* Launch stream (cudaStream_t; NULL = the context's own stream).  The reference uses the
 * default stream throughout (FD2DGPU.cuh:282 stream parameters receive 0). */
int ds2d_set_stream(ds2d_ctx *ctx, void *stream);

/* FD2DGPU_ELASTIC::GPUbufferVPVS (FD2DGPU.cu:1310).  rho may be NULL: the reference hard-wires
 * rho = 2000 (FD2DGPU.cu:1121). */
int ds2d_set_models(ds2d_ctx *ctx, const float *vp, const float *vs, const float *rho);
/* Source wavelet, nt samples (constructor argument `sou`, FD2DGPU.cu:55; main.cpp:1476). */
int ds2d_set_wavelet(ds2d_ctx *ctx, const float *wavelet);
/* FD2DGPU_ELASTIC::GPUbufferM (FD2DGPU.cu:1316): reflectivity images used by the Born source. */
int ds2d_set_image(ds2d_ctx *ctx, const float *image_pp, const float *image_ps);

/* Background forward modelling of n shots (FD2DGPU.cu:4398-4400 addS + born_modeling mode 0),
 * recording vz / vx at the receivers after every step.  rec_* receive [sum ntr][nt]. */
int ds2d_forward(ds2d_ctx *ctx, const ds2d_shot *shots, int n, float *rec_vz, float *rec_vx);

/* Reference-mode ELSRTM of n shots: ELSRTM_ROT_EXP_IMAGE_SINGLESHOT (FD2DGPU.cu:4184) per shot,
 * with record_copytoGPU (:3537) and bufferVpVsHtoD (:1336) folded in.  obs_* are the observed
 * records [sum ntr][nt], in host or device memory (copied with unified addressing; the reference
 * takes host records, record_copytoGPU).  Gradients accumulate in the context's seven images
 * (read them with ds2d_read_images); *misfit accumulates like the reference's double& argument.
 * lm_* / res_* may be NULL; when given they receive Lm + Lm2 and the injected adjoint source
 * (host arrays). */
int ds2d_elsrtm(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *obs_vz,
                const float *obs_vx, int iter, double *misfit, float *lm_vz, float *lm_vx,
                float *res_vz, float *res_vx);

/* Elastic RTM of n shots: background forward pass, then interior reconstruction
 * (FD2DGPU.cu:4769-4772), adjoint propagation of adj_* injected at the receivers (:3306,
 * stack = true; :4775-4778) and zero-lag imaging (:3245 doimage_gradient, :3235 doimage_illum)
 * into images 0 (pp), 1 (ps) and 2 (illumination).  adj_* are host arrays [sum ntr][nt]. */
int ds2d_rtm(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *adj_vz,
             const float *adj_vx);
/* Same as ds2d_rtm with adj_* already in device memory (no host copies). */
int ds2d_rtm_device(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *adj_vz_dev,
                    const float *adj_vx_dev);

/* FD2DGPU_ELASTIC::imagebuffer_resettozero (FD2DGPU.cu:3478): copies the seven accumulated
 * images (pp_grad, ps_grad, illumination, b_pp, b_ps, b_pp2, b_ps2; each [allnx][allnz]) to the
 * host arrays that are not NULL, then zeroes them when reset != 0. */
int ds2d_read_images(ds2d_ctx *ctx, float *const images[7], int reset);

/* The same read-out into DEVICE arrays (no counterpart in the reference, whose gradients cross
 * to the host and MPI_Reduce there, main.cpp:1038-1060): the non-NULL images are copied device
 * to device on the context stream, then zeroed when reset != 0; returns without synchronising.
 * For one process per GPU, the caller all-reduces those arrays in place over NCCL. */
int ds2d_read_images_device(ds2d_ctx *ctx, float *const images[7], int reset);

/* Cell-updates performed by the last ds2d_forward / ds2d_elsrtm / ds2d_rtm call (padded cells x
 * steps x propagations), for throughput reporting. */
double ds2d_last_cell_updates(const ds2d_ctx *ctx);

/* Number of kernel launches issued by the last forward / elsrtm / rtm call. */
long long ds2d_last_launches(const ds2d_ctx *ctx);

/* Acoustic Born operator pair and CG-LSRTM (an extension of the path; the reference ships unused
 * CG helpers, main.cpp:1224-1320 sjcgsolver / FD2DGPU.cu:4885 ELSRTM_CALCULATE_ALPHA, and runs
 * NCC + Adam instead).  The acoustic scheme is the elastic one with mu = 0 (pass vs = 0 to
 * ds2d_set_models); the context must use DS2D_BOUNDARY_RANDOM (undamped grid, exact time
 * reversal).  m / grad are [allnx][allnz]; records [sum ntr][nt]; these arrays may be in host
 * or device memory (copies use unified addressing).
 *   ds2d_ac_born      d = L m  (scattered vz, vx; Born source of add_born_source with mu = 0)
 *   ds2d_ac_born_adj  g = L^T d, the exact discrete transpose of ds2d_ac_born
 *   ds2d_ac_normal    img = L^T L m: the RTM image of the Born data of m, records kept on the
 *                     device (training pairs of the learned preconditioner)
 *   ds2d_lsrtm        CGLS on ||L m - d||^2 from m = 0 with FP64 inner products and step
 *                     lengths; stops after niter iterations or when ||d - L m|| / ||d|| <=
 *                     target; resid[k] receives that ratio after iteration k.
 *   ds2d_lsrtm_pcg    the same problem by flexible preconditioned CG: direction z = P(L^T r)
 *                     with P the U-Net `net` (NULL: P = I, plain CG), explicit L^T L-conjugation
 *                     against the last "pcg_m" directions (default 8; flexible CG, FCG(M)) and
 *                     the exact step <r, L p> / ||L p||^2; when an iteration with the
 *                     network reduces the residual by less than the "pcg_switch" option (per
 *                     mille, default 970) the solver restarts as plain CG from the current
 *                     iterate.  elapsed_ms[k] (may be NULL) is the wall time from the call's start
 *                     to the end of iteration k. */
int ds2d_ac_born(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *m, float *rec_vz,
                 float *rec_vx);
int ds2d_ac_born_adj(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *rec_vz,
                     const float *rec_vx, float *grad);
int ds2d_lsrtm(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *obs_vz,
               const float *obs_vx, int niter, double target, float *m_out, double *resid,
               int *iters_done);
int ds2d_ac_normal(ds2d_ctx *ctx, const ds2d_shot *shots, int n, const float *m, float *img);
struct ds2d_unet;
int ds2d_lsrtm_pcg(ds2d_ctx *ctx, struct ds2d_unet *net, const ds2d_shot *shots, int n,
                   const float *obs_vz, const float *obs_vx, int niter, double target,
                   float *m_out, double *resid, double *elapsed_ms, int *iters_done);

/* FP64 inner product <a, b> of two float vectors of n elements in device memory, the
 * reduction the CG-LSRTM uses for its dot products and step lengths (the reference sums its CG
 * products in float on the host, main.cpp:1232-1276).  Per-block partial sums go to scratch
 * owned by the context, then one block adds them in a fixed order, so the result is
 * deterministic.  Runs on the context stream and returns after the result is on the host. */
int ds2d_dot_f64(ds2d_ctx *ctx, const float *a, const float *b, long long n, double *result);

/* The same FP64 inner product with no context and no device allocation (no counterpart in the
 * reference, which has no device-side reduction).  For callers that cannot allocate device
 * memory when they need the product: a host framework that owns the device memory budget, a
 * caller with no ds2d context, or one running with the HBM already full.  The partial sums live
 * in a static device array of the library (256 KiB per device), so:
 *  - n is limited to 536,870,912 elements (32768 partial sums of 16384 elements each); a larger
 *    n returns DS2D_E_ARG with a message, and nothing is launched;
 *  - the first call in a CUDA context of a device looks up that array's address with the device
 *    current (and may load the library's module there), so make it before any stream capture
 *    on that device; the address is cached per device with the context it belongs to, and a
 *    call from a different context (a non-primary one, or the primary context re-created after
 *    cudaDeviceReset) looks it up again;
 *  - calls on the same device that overlap in time (other host threads, or streams whose work
 *    runs concurrently) share the array and race: serialise them.
 * Runs on `stream` (NULL = the legacy default stream) of the current device and returns after
 * the result is on the host.  Errors are reported by ds2d_last_error(NULL).  Summation order
 * differs from ds2d_dot_f64 (contiguous chunks instead of a grid stride), so the two agree to
 * FP64 rounding, not bit for bit. */
int ds2d_dot_f64_noalloc(const float *a, const float *b, long long n, void *stream,
                         double *result);

/* Gradient band-pass filter, replacing the reference's bandpass_filter (FD2DGPU.cu:4125-4182,
 * which main.cpp:1074-1089 applies to the summed gradients when enabled): each [nx][nz] image
 * (z fastest) is transformed to the 2D spectrum in FP64, multiplied by the Gaussian band-pass of
 * construct_gaussian_bandpass_filter (FD2DGPU.cu:4038-4077) with low cut-off z1 (0 = low-pass)
 * and high cut-off z2, and transformed back, reproducing the reference's quadrant swaps and its
 * complex (k, k) multiply.  x1, x2 are accepted for the reference's signature and unused, as in
 * its live filter.  ds2d_bandpass_filter takes host arrays (copied in and out, like the
 * reference); ds2d_bandpass_filter_device filters device arrays in place on `stream`.  Either
 * image pointer may be NULL.  Both allocate their scratch per call (two DFT matrices and three
 * work planes, about 16 (nx^2 + nz^2 + 3 nx nz) bytes).  Errors via ds2d_last_error(NULL). */
int ds2d_bandpass_filter(int nx, int nz, int x1, int x2, int z1, int z2, float *grad_pp,
                         float *grad_ps);
int ds2d_bandpass_filter_device(int nx, int nz, int x1, int x2, int z1, int z2, float *grad_pp,
                                float *grad_ps, void *stream);

/* Tuning knobs (no counterpart in the reference, whose launch shape is fixed at 32x32 blocks,
 * FD2DGPU.cuh:8-9): "fused" (1 = single-pass fused time step, 0 = one launch per half step),
 * "xr" (rows marched by one CTA of the fused kernels), "ring" (cp.async prefetch ring depth of
 * the fused kernels: 0 off, 1 default, or 2 / 4 / 8), "occ" (0 / 1: register budget for 6 / 8
 * forward and 3 / 4 backward CTAs per SM), "cta" (threads per CTA of the ring kernels: 128,
 * 192, or 0 = the one whose z-strips leave fewer threads idle for this grid; 192 needs ring 4 and
 * occ 0), "graph" (0 / 1: capture batches in CUDA graphs),
 * "adjoint_born" (see ds2d_elsrtm), "pcg_switch" and "pcg_m" (1..15, see ds2d_lsrtm_pcg).
 * Pair-blocked bulk-copy kernels (random boundary; two z-columns per thread, rows fed by
 * cp.async.bulk into an mbarrier ring): "pair" (0 off, 1 forward and backward RTM steps, 2 the
 * forward step only: the default), "pair_fcta" (forward CTA width 64 / 256, 0 = 256), "pair_cta" (backward
 * 64 / 160 / 256, 0 = 64), "pair_split" (0 / 1: backward in one or two launches), "pair_xr" (rows
 * per CTA, 0 = the count that fills the SMs' waves best), "ac_pair" (0 / 1: acoustic forward
 * steps of the Born pair on k_ac_pair) and "ac_pair_cta" (128 / 192 / 256, 0 = the width with the
 * fewest threads per grid row).  "ac_ckpt" (K, 0 = off; PML acoustic L^T): keep a snapshot of
 * the whole background state every K steps, in the strip precision with one FP32 scale per field,
 * shot and snapshot, and replay each K-step segment from its snapshot with strips before
 * reversing it: snapshots plus K steps of strips instead of nt steps of strips, for one more
 * forward propagation per L^T.  Random-boundary RTM steps: "tb" (K = 1-4 forward time steps
 * per launch, default 2; 0 = one step per launch on the pair / ring kernels), "tb_cta" (256 / 512,
 * 0 = automatic), "tb_bulk" (1 = operand rows by bulk copy at depth 1-2, the default); the backward step
 * "bwd_bulk" (1 = operand rows by bulk copy, the copy issue spread over all warps: the default;
 * 0 = per-thread cp.async), "bwd_cta" (threads per CTA of the bulk-copy step: 128 / 192 / 256,
 * 0 = the width with the fewest threads per grid row), "bwd_1b" (1 = one barrier per row step:
 * the default; 0 = two), "bwd_ws" (0 off, or 96 / 128 / 192 threads per role of the
 * warp-specialised step). */
int ds2d_set_option(ds2d_ctx *ctx, const char *key, long long value);

/* Profiling (no counterpart in the reference, which has only a commented-out host timer,
 * FD2DGPU.cu:3554-3583): when enabled, every launch is bracketed by CUDA events on the launch
 * stream.  ds2d_profile_report writes one line per kernel, "name launches total_ms
 * algorithmic_bytes", for the launches since the last report, and clears them. */
int ds2d_profile(ds2d_ctx *ctx, int enable);
int ds2d_profile_report(ds2d_ctx *ctx, char *buf, int len);

/* ---- Learned preconditioner: image-domain U-Net (no counterpart in the reference) --------
 * Maps an RTM image to an estimate of the reflectivity (an approximate inverse Hessian of the
 * Born operator) to precondition CG-LSRTM.  4-level encoder-decoder, `base` (32) channels at the
 * first level doubling per level, conv3x3 + ReLU pairs, 2x2 average pooling, nearest 2x
 * upsampling with skip concatenation, 1x1 output convolution; BF16 activations and weights on
 * the tensor cores with FP32 accumulation and FP32 master weights.  Images are FP32 [n][h][w] in
 * device memory with h and w multiples of 8.  Parameters are one flat FP32 vector: per layer (in
 * the order e1a e1b e2a e2b e3a e3b e4a e4b d3a d3b d2a d2b d1a d1b out) the weights
 * [ky][kx][cout][cin] followed by the biases [cout]. */
typedef struct ds2d_unet ds2d_unet;
int ds2d_unet_create(int base, int max_n, int max_h, int max_w, int device, ds2d_unet **out);
int ds2d_unet_destroy(ds2d_unet *net);
const char *ds2d_unet_last_error(const ds2d_unet *net); /* NULL: error of the last create */
int ds2d_unet_set_stream(ds2d_unet *net, void *stream);
long long ds2d_unet_num_params(const ds2d_unet *net);
int ds2d_unet_set_params(ds2d_unet *net, const float *params, long long n); /* host; resets Adam */
int ds2d_unet_get_params(ds2d_unet *net, float *params, long long n);                /* host */
/* y = net(x), both device [n][h][w] FP32. */
int ds2d_unet_forward(ds2d_unet *net, const float *x, float *y, int n, int h, int w);
/* Mean-squared-error loss of net(x) against target (device arrays) and the gradient of every
 * parameter (kept on the device for ds2d_unet_adam_step; copied to grads_host when non-NULL). */
int ds2d_unet_loss_grad(ds2d_unet *net, const float *x, const float *target, int n, int h, int w,
                        double *loss, float *grads_host);
/* One Adam step (bias-corrected) with the gradients of the last ds2d_unet_loss_grad. */
int ds2d_unet_adam_step(ds2d_unet *net, float lr, float beta1, float beta2, float eps);
/* "tcgen05" = 1 (default) runs the 3x3 convolutions (forward, backward-data and weight gradient)
 * on the 5th-generation tensor cores with TMEM accumulators; 0 runs all three on mma.sync.
 * "tcgen05_wgrad" = 0 keeps only the weight gradient on mma.sync (default 1).  "tcgen05_tma" = 1
 * (default) feeds the tcgen05 convolution by tiled bulk-tensor loads through a ring of
 * "tcgen05_stages" = 2 (default) or 3 stages; 0 stages the operands through the threads.
 * "tcgen05_rows" = 1, 2 or 4 (default) output rows per CTA (the bulk-tensor kernel takes 2 or 4;
 * the thread-staged one keeps 2 for 128-channel tiles).  "tcgen05_wgrad_tma" = 1 (default) loads
 * the weight gradient's operands MN-major by bulk-tensor boxes; 0 transposes them through the
 * threads. */
int ds2d_unet_set_option(ds2d_unet *net, const char *key, long long value);

#ifdef __cplusplus
}
#endif
#endif
