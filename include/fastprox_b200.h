/*
 * fastprox_b200.h -- the image total-variation entry points of fastprox's
 * plain-C ABI (ABI version 1), served by sm_100a CUDA kernels.
 *
 * A drop-in for the image-TV subset of the reference library: the types,
 * enum values, structure layouts and function signatures below are those of
 * the reference's include/fastprox.h, so a caller compiled against that
 * header links against libfastprox_b200.so unchanged. Arrays on a CUDA
 * device (FP_DEVICE_CUDA, DLPack's kDLCUDA) are solved in place on that
 * device; arrays in host memory (FP_DEVICE_CPU) are staged through the
 * workspace's device buffers and solved on the GPU as well. There is no CPU
 * solver behind these entry points: without a usable GPU they return
 * FP_EDEVICE.
 *
 * Every function is extern "C", returns fp_status (or a plain value), and
 * lets no C++ exception escape.
 */
#ifndef FASTPROX_B200_H
#define FASTPROX_B200_H

#include <stddef.h>
#include <stdint.h>

#define FP_VERSION_MAJOR 1
#define FP_VERSION_MINOR 0
#define FP_VERSION_PATCH 6
#define FP_ABI_VERSION 1
#define FP_MAX_NDIM 32

#define FP_API __attribute__((visibility("default")))

#ifdef __cplusplus
extern "C" {
#endif

/* Same values as the reference's fp_dtype / fp_device / fp_status
 * (include/fastprox.h:52-80). */
typedef enum { FP_F32 = 1, FP_F64 = 2, FP_I8 = 3, FP_I32 = 4, FP_I64 = 5 } fp_dtype;
typedef enum { FP_DEVICE_CPU = 0, FP_DEVICE_CUDA = 2 } fp_device;

/* Strided n-d array; strides in elements (NULL = C order); never freed by
 * the library (include/fastprox.h:61-68). */
typedef struct {
    void          *data;
    fp_dtype       dtype;
    int            ndim;
    const int64_t *shape;
    const int64_t *strides;
    fp_device      device;
} fp_array;

typedef enum {
    FP_OK = 0,
    FP_EINVAL,
    FP_EDTYPE,
    FP_ESHAPE,
    FP_ENOMEM,
    FP_ENOTCONV,
    FP_EPARAM,
    FP_EINTERNAL,
    FP_EDEVICE
} fp_status;

typedef struct fp_op fp_op;
typedef struct fp_workspace fp_workspace;

/* include/fastprox.h:93-103. threads is ignored on the device. */
typedef struct {
    int    axis;
    int    threads;
    double tol;
    int    max_iter;
    int    tie;
    int    keep_structure;
} fp_options;

/* include/fastprox.h:105-109. */
typedef struct {
    double  gap;
    int     iters;
    int64_t ties;
} fp_info;

/* Replaces fp_options_init, include/fastprox.h:113. Defaults: axis -1,
 * threads 0, tol 1e-6, max_iter 1000, tie 0, keep_structure 0. */
FP_API void fp_options_init(fp_options *opt);

/* Operator constructors: replace include/fastprox.h:322, :332, :343, :352
 * (fp_op_tv_aniso, fp_op_tv_aniso_weighted, fp_op_tv_iso,
 * fp_op_tv_iso_weighted). Same parameter rules and errors: ndim 2 or 3
 * (FP_EPARAM otherwise); axis_weights NULL, length 1 or ndim, finite and
 * >= 0; pixel weights of the image shape, edge weights of shape
 * (ndim, image shape), finite and >= 0. Parameter arrays must be host
 * arrays (they are copied). */
FP_API fp_status fp_op_tv_aniso(int ndim, const fp_array *axis_weights, fp_op **out);
FP_API fp_status fp_op_tv_aniso_weighted(int ndim, const fp_array *axis_weights,
                                         const fp_array *edge_weights, fp_op **out);
FP_API fp_status fp_op_tv_iso(int ndim, const fp_array *axis_weights, fp_op **out);
FP_API fp_status fp_op_tv_iso_weighted(int ndim, const fp_array *axis_weights,
                                       const fp_array *pixel_weights, fp_op **out);

/* Replace include/fastprox.h:392-394. */
FP_API void        fp_op_free(fp_op *op);
FP_API int64_t     fp_op_nparams(const fp_op *op);
FP_API const char *fp_op_name(const fp_op *op);

/* Replaces include/fastprox.h:411-413. Every byte of device memory the
 * calls on this workspace use is allocated here, on the calling thread's
 * current device (FP_DEVICE_CUDA like) or on device 0 (FP_DEVICE_CPU like,
 * whose calls then stage host arrays through it). */
FP_API fp_status fp_workspace_create(const fp_op *op, const fp_array *like,
                                     const fp_options *opt, fp_workspace **out);
FP_API void      fp_workspace_free(fp_workspace *ws);

/* Replace include/fastprox.h:426-428: the dual (ndim, *x.shape) of the last
 * call, a seed for the next one, and warm starts from the previous call. */
FP_API fp_status fp_workspace_get_dual(const fp_workspace *ws, fp_array *out);
FP_API fp_status fp_workspace_set_dual(fp_workspace *ws, const fp_array *dual);
FP_API fp_status fp_workspace_set_warm(fp_workspace *ws, int on);

/* Replace include/fastprox.h:437-438 (derivative conjugate gradients). */
FP_API fp_status fp_workspace_set_deriv_tol(fp_workspace *ws, double tol, int max_iter);
FP_API fp_status fp_workspace_deriv_info(const fp_workspace *ws, double *residual, int *iters);

/* Replaces include/fastprox.h:599-601. Stops each image when its duality gap
 * is at most tol |x|^2 / 2; FP_ENOTCONV after max_iter with the last iterate
 * written. Waits for the stream (it reads per-image flags between groups of
 * iterations). */
FP_API fp_status fp_prox(const fp_op *op, double gamma, const fp_array *x,
                         fp_array *out, const fp_options *opt,
                         fp_workspace *ws, fp_info *info);

/* Replaces include/fastprox.h:613-614: one step per image (gamma has x's
 * batch shape, host or device memory). */
FP_API fp_status fp_prox_steps(const fp_op *op, const fp_array *gamma, const fp_array *x,
                               fp_array *out, const fp_options *opt, fp_workspace *ws);

/* Replaces include/fastprox.h:637-639 for the TV operators (positively
 * homogeneous: the result is y - prox_g(y), for every sigma > 0; y for
 * sigma = 0). */
FP_API fp_status fp_prox_conj(const fp_op *op, double sigma, const fp_array *y,
                              fp_array *out, const fp_options *opt,
                              fp_workspace *ws, fp_info *info);

/* Replace include/fastprox.h:646-654 and :779-780: derivatives at the point
 * kept by the last prox call with keep_structure, isotropic or anisotropic
 * TV. theta = the k axis weights, then the pixel weights (isotropic) or edge
 * weights (anisotropic, k x shape) in C order (fp_op_nparams entries);
 * gparams and dparams may be host or device arrays, float32 or float64,
 * ndim <= 1. */
FP_API fp_status fp_jvp(const fp_op *op, const fp_workspace *ws,
                        const fp_array *dx, double dgamma,
                        const fp_array *dparams, fp_array *dout);
FP_API fp_status fp_vjp(const fp_op *op, const fp_workspace *ws,
                        const fp_array *g, fp_array *gx, double *ggamma,
                        fp_array *gparams);
FP_API fp_status fp_vjp_device(const fp_op *op, const fp_workspace *ws, const fp_array *g,
                               fp_array *gx, fp_array *ggamma, fp_array *gparams);

/* Replace include/fastprox.h:510-512: the kink mask of the kept point
 * (FP_I8, x's shape, any strides, host or device; NULL for the count only)
 * at tolerance tol and the number of entries at a kink: isotropic TV 1 where
 * |(W D z)_p| <= tol and |u_p| >= gamma alpha_p - tol, anisotropic TV bit a
 * at an edge (p, p + e_a) with |z jump| <= tol and |p_e| >= lam_e - tol
 * (zero bounds are never kinks). set_branch (anisotropic TV; FP_EINVAL for
 * isotropic TV) picks at each kink the piece the derivatives differentiate:
 * side -1 joins the edge's two ends, +1 keeps them apart, 0 the default; it
 * holds until the next prox call or a call with side NULL. */
FP_API fp_status fp_workspace_kinks(const fp_workspace *ws, double tol, fp_array *mask,
                                    int64_t *count);
FP_API fp_status fp_workspace_set_branch(fp_workspace *ws, const fp_array *side, double tol);

/* Replace include/fastprox.h:514-579: the structure of the derivative at the
 * kept point. Units are the images; every entry of a TV solution is FREE,
 * with sign +1, in a region (its label, numbered in order of first entries
 * within its image; -1 and sign 0 in an image holding a NaN, whose region
 * count is -1); no linear constraint. After fp_prox_conj at sigma = 0 every
 * entry is ZERO, without regions. The reference answers these on host
 * workspaces only (FP_EINVAL on a device one); here every workspace is
 * answered, the outputs host or device arrays. */
typedef enum {
    FP_ENTRY_FREE  = 0,
    FP_ENTRY_ZERO  = 1,
    FP_ENTRY_LOWER = 2,
    FP_ENTRY_UPPER = 3
} fp_entry_state;

typedef enum {
    FP_STRUCT_NONE      = 0,
    FP_STRUCT_PROJECTOR = 1, /* anisotropic TV: the average over each region */
    FP_STRUCT_WEIGHTED  = 2,
    FP_STRUCT_CURVED    = 3  /* isotropic TV: range span M, not a projector */
} fp_struct_kind;

FP_API fp_status fp_op_struct_kind(const fp_op *op, int *kind);
FP_API fp_status fp_workspace_units(const fp_workspace *ws, int64_t *count, int64_t *size);
FP_API fp_status fp_workspace_states(const fp_workspace *ws, fp_array *state, int64_t *nfixed);
FP_API fp_status fp_workspace_regions(const fp_workspace *ws, fp_array *labels, fp_array *sign,
                                      int64_t *nregions, int64_t count);
FP_API fp_status fp_workspace_constraint(const fp_workspace *ws, fp_array *coef, int8_t *active,
                                         int64_t count);

/* Replaces include/fastprox.h:769: whether every image's derivative is
 * exact (anisotropic TV: its polish certified the regions; isotropic TV:
 * without smoothing) and the largest curvature cap mu of the isotropic
 * derivative, in the units of x. */
FP_API fp_status fp_workspace_deriv_exact(const fp_workspace *ws, int *exact, double *smoothing);

/* Replaces include/fastprox.h:770-771: the kept call solved again from its
 * saved input, warm from its dual, to tol within max_iter; the derivatives,
 * the dual and the call's results then describe the refined point (the first
 * call's z is not changed). out (x's shape and dtype, may be NULL) receives
 * the refined result; FP_ENOTCONV as fp_prox. */
FP_API fp_status fp_workspace_refine(const fp_op *op, fp_workspace *ws, double tol, int max_iter,
                                     fp_array *out, fp_info *info);

/* Replace include/fastprox.h:712 and :718. */
FP_API int       fp_device_available(fp_device dev);
FP_API fp_status fp_op_device_check(const fp_op *op, fp_device dev, int *row_parallel_only);

/* Replace include/fastprox.h:724-725. */
FP_API fp_status fp_workspace_set_stream(fp_workspace *ws, void *stream);
FP_API fp_status fp_workspace_get_stream(const fp_workspace *ws, void **stream);

/* Replace include/fastprox.h:732 and :773-774. */
FP_API fp_status fp_workspace_info(const fp_workspace *ws, fp_info *info);
FP_API fp_status fp_workspace_image_info(const fp_workspace *ws, double *gaps, int *iters,
                                         double *zerrs, int64_t count);

/* Replace include/fastprox.h:782-789. */
FP_API const char *fp_strerror(fp_status s);
FP_API int         fp_abi_version(void);
FP_API const char *fp_version_string(void);
FP_API int         fp_default_threads(void);

/* ------------------------------------------------------------------------
 * Extensions of this library (no counterpart in the reference ABI).
 * ---------------------------------------------------------------------- */

/* Counters of the last prox call on ws: the kernels it launched (set-up,
 * iterations, finalisation) and the step launches alone. For benchmarks and
 * tests; FP_EINVAL before a call. */
FP_API fp_status fp_b200_workspace_stats(const fp_workspace *ws, int64_t *kernel_launches,
                                         int64_t *step_launches);

/* Device time of the isotropic step launches of the next prox calls on ws:
 * with on = 1, each step launch of a call is bracketed by a pair of events on
 * the workspace's stream (up to 4096 launches per call), which serialises the
 * launches and adds a little to the call. fp_b200_workspace_step_times then
 * gives the last call's total milliseconds and launches of one kind: 0 single
 * iterations, 1 two iterations per launch, 2 two iterations the second of
 * which carries the gap check, 3 four iterations per launch (the fourth with
 * the gap check). For benchmarks. */
FP_API fp_status fp_b200_workspace_time_steps(fp_workspace *ws, int on);
/* The last fp_vjp (or fp_vjp_device) on ws, per image, before its sums over
 * the batch: ggamma[b] the gradient of image b's step, gweights[b k + a] that
 * of axis weight a from image b (k = the operator's ndim); either may be NULL.
 * For callers with one step per image (fp_prox_steps), whose gradient
 * fp_vjp returns summed. count must be the batch size (FP_EINVAL otherwise, or
 * before any fp_vjp). No counterpart in the reference ABI. */
FP_API fp_status fp_b200_vjp_images(const fp_workspace *ws, double *ggamma, double *gweights, int64_t count);
FP_API fp_status fp_b200_workspace_step_times(const fp_workspace *ws, int kind, double *ms, int64_t *launches);

/* Workspaces take their device memory from a stream-ordered pool per device
 * and their pinned host memory from a cache, so creating and freeing one
 * (once per call when fp_prox gets ws = NULL) never synchronises the whole
 * device. Freed memory stays cached for the next workspace; this returns it
 * all to the driver. */
FP_API void fp_b200_release_cached(void);

/* Ragged batches and continuous batching (no counterpart in the reference,
 * whose calls take one array shape each). An fp_b200_batch solves isotropic
 * 2D TV (an operator from fp_op_tv_iso, unit or axis weights, no pixel
 * weights) on images of any sizes at once: admitted images share one set of
 * kernel launches, each image stops on its own gap, and images can be
 * admitted between calls to fp_b200_batch_run while others iterate.
 * Results are the same bits whatever else is in the batch.
 *
 * create: capacity for max_images images and max_pixels pixels in all, every
 * byte of device memory allocated here, on the current device; dtype FP_F32
 * or FP_F64 (the images' dtype). admit: x and z are device pointers to
 * contiguous (height, width) arrays (z may be x), copied in now, solved by
 * later runs; tol and max_iter as in fp_prox, per image; FP_ENOMEM when no
 * slot or not enough contiguous pixels are free (admit again after a run has
 * finished others). run: repeats `steps` steps of every live image (as a
 * captured CUDA graph; a step advances an image by one iteration, or by four
 * on float images whose width is a multiple of 4, in two launches of two
 * iterations each) until at least one image has finished or none is live;
 * writes the finished images' z, and their slots, gaps and iterations (a
 * negative count: stopped at max_iter) into arrays of max_images entries;
 * *nlive, the images still iterating. max_chunks > 0 bounds the chunks of
 * `steps` steps one run may take (it may then return with none
 * finished, so that a serving loop can admit new images in between). All
 * calls on one batch run on its stream (set_stream; NULL by default) and
 * must not overlap. */
typedef struct fp_b200_batch fp_b200_batch;
FP_API fp_status fp_b200_batch_create(const fp_op *op, int64_t max_images, int64_t max_pixels, int dtype,
                                      fp_b200_batch **out);
FP_API void      fp_b200_batch_free(fp_b200_batch *bt);
FP_API fp_status fp_b200_batch_set_stream(fp_b200_batch *bt, void *stream);
/* Whether runs replay captured CUDA graphs (the default) or launch their
 * kernels one by one; a capture that fails (other threads using the device)
 * falls back to launches by itself. */
FP_API fp_status fp_b200_batch_set_graphs(fp_b200_batch *bt, int on);
/* Rows per tile of images admitted from now on (0: chosen from the image
 * height); the tuner sets it. */
FP_API fp_status fp_b200_batch_set_rows(fp_b200_batch *bt, int rows);
/* Quad launches (four iterations per launch) for the float images of rows of a
 * multiple of 4 pixels admitted from now on: on (default) or off, and the rows
 * of a quad tile (0 keeps the current, 32 by default). For the tuner. */
FP_API fp_status fp_b200_batch_set_quads(fp_b200_batch *bt, int on, int rows);
FP_API fp_status fp_b200_batch_admit(fp_b200_batch *bt, const void *x, int64_t height, int64_t width, double gamma,
                                     double tol, int max_iter, void *z, int *slot);
FP_API fp_status fp_b200_batch_run(fp_b200_batch *bt, int steps, int max_chunks, int *finished, double *gaps,
                                   int *iters, int *nfinished, int *nlive);
FP_API fp_status fp_b200_batch_stats(const fp_b200_batch *bt, int64_t *kernel_launches, int64_t *steps,
                                     int64_t *free_pixels);

/* Huber-smoothed TV, the reference's planned first analysis prior (its
 * ROADMAP.md, "Stage 1, Huber-smoothed TV": fp_op_tv_iso_huber,
 * fp_op_tv_aniso_huber; designed there, not in its code). Isotropic:
 * g(z) = sum_p alpha_p h(|(W D z)_p|); anisotropic:
 * g(z) = sum_a sum_p beta[a, p] h(|w_a (D_a z)_p|); h the Huber function of
 * fp_op_huber (include/fastprox.h:129-131) with smoothing delta, finite and
 * > 0 (FP_EPARAM otherwise). Weights, shapes and errors as fp_op_tv_iso[_weighted]
 * and fp_op_tv_aniso[_weighted] (pixel_weights / edge_weights may be NULL).
 * fp_prox / fp_prox_steps solve it by dual FISTA with a constant momentum
 * (the dual is strongly convex: linear convergence), stopped on the same
 * duality gap, |z - z*|^2 <= 2 gap; the dual returned is q with
 * x - z = sum_a w_a D_a^T q_a. theta = the axis weights, the pixel or edge
 * weights, then delta. The derivatives (fp_vjp, fp_jvp, the structure
 * queries) are not built for it: FP_EINVAL. */
FP_API fp_status fp_b200_op_tv_iso_huber(int ndim, const fp_array *axis_weights, const fp_array *pixel_weights,
                                         double delta, fp_op **out);
FP_API fp_status fp_b200_op_tv_aniso_huber(int ndim, const fp_array *axis_weights, const fp_array *edge_weights,
                                           double delta, fp_op **out);

/* Isotropic 2D TV prox of a small float32 batch without allocating any
 * memory. No counterpart in the reference ABI.
 *
 * For callers that must not allocate device memory: a custom operator inside
 * another runtime that plans all device memory ahead of time (an inference
 * server with a fixed memory budget), a caching allocator's out-of-memory
 * handler, or latency-bound code that may not call cudaMalloc because it can
 * synchronise the whole device. fp_prox needs a workspace, and creating one
 * allocates; this entry point takes its scratch from a fixed array inside the
 * library instead (about 48 MB). It calls no cudaMalloc, cudaFree or other
 * allocating routine.
 *
 * When the array is reserved: the CUDA runtime loads the library's isotropic
 * kernels, and reserves the array with them, on a device the first time any
 * of them runs there (lazy module loading): the first call of this entry
 * point, or the first isotropic fp_prox, on that device. That first call can
 * therefore fail with FP_EDEVICE when the device is out of memory. A caller
 * that must never allocate makes one small call on each device it uses at
 * start-up (before any stream capture); later calls reserve nothing more. The
 * array then stays reserved on that device until the process exits.
 *
 * x and z: device pointers on the calling thread's current device to
 * contiguous (batch, height, width) float32 arrays; z may equal x. Unit axis
 * weights, no pixel weights; gamma, tol and max_iter as in fp_prox. stream: a
 * cudaStream_t (NULL for the legacy default stream); the call waits for it.
 * gaps, iters: host arrays of batch entries for the per-image duality gap and
 * iterations, or NULL. Limits: batch <= 64 and batch * height * width <= 2^20
 * (FP_ESHAPE beyond them). Returns FP_OK, FP_ENOTCONV, FP_EINVAL (an image
 * holding +-Inf), FP_EPARAM or FP_EDEVICE. The results are fp_prox's for the
 * same input (the same launch shapes and partial sums).
 *
 * Every call shares the one scratch array, which keeps the last call's
 * contents: calls that overlap on the GPU (from two host threads, or on two
 * streams) race and corrupt each other's results; serialise them. The
 * array's device address is looked up on each call. */
FP_API fp_status fp_b200_tv_iso_noalloc(const float *x, float *z, int64_t batch, int64_t height, int64_t width,
                                        double gamma, double tol, int max_iter, void *stream, double *gaps,
                                        int *iters);

#ifdef __cplusplus
}
#endif

#endif /* FASTPROX_B200_H */
