/*
 * lya2pcf B200 pair-binning library: C ABI.
 *
 * One context per thread of control; every call returns an int status
 * (LYA_OK == 0) and never throws or exits; lya_last_error() describes the most
 * recent failure.  Host buffers are caller-owned and only read or written
 * during the call; the library owns all device memory of a context and runs
 * every kernel on the context's own stream.
 *
 * Each entry point names the reference routine whose role it takes
 * (lya2pcf, file:line).
 */
#ifndef LYA2PCF_H
#define LYA2PCF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LYA_OK 0
#define LYA_ERR_ARG 1      /* bad argument: null pointer, size, shape, option */
#define LYA_ERR_CUDA 2     /* a CUDA runtime call failed */
#define LYA_ERR_ALLOC 3    /* device or host allocation failed */
#define LYA_ERR_STATE 4    /* call out of order (e.g. run before upload) */
#define LYA_ERR_DATA 5     /* input data violates a documented requirement */
#define LYA_ERR_GUARD 6    /* guard band narrower than the FP32 error bound */
#define LYA_ERR_DEVICE 7   /* a kernel reported an internal error flag */

/* kernels of lya_corr_run */
#define LYA_KERNEL_FP32_GUARDED 0 /* FP32 diagonal-run kernel, FP64 recheck in the guard band */
#define LYA_KERNEL_FP64_DIAGONAL 1 /* same walk, FP64 geometry and run sums */
#define LYA_KERNEL_FP64_PLAIN 2    /* every pixel pair, FP64, one shared atomic per quantity */

/* histogram quantities, in output order: sum w1w2, sum dw1dw2, sum w1w2*rp,
 * sum w1w2*rt, sum w1w2*(z1+z2)/2 */
#define LYA_NQ 5

typedef struct lya_ctx lya_ctx;

typedef struct {
  int32_t kernel;          /* LYA_KERNEL_* */
  double guard;            /* guard half-width around bin edges, Mpc/h (FP32 kernel) */
  int32_t warps_per_block; /* 0 = default (16) */
  int32_t blocks_per_sm;   /* 0 = default (1) */
  int32_t slot_begin;      /* restrict the run to pairs whose first forest's */
  int32_t slot_end;        /* slot is in [slot_begin, slot_end); 0,0 = all    */
  int32_t variant;         /* diagonal walk: 0 = default (FP32: the lean walk --
                              two diagonals per lane, bin tests on the FP32 pixel
                              coordinates -- for pairs of sorted forests with
                              0 <= dc < 1e6, walk 2 for the others; FP64: one
                              diagonal per lane), 1 = one diagonal per lane,
                              2 = two diagonals per lane, 3 = same as 0 */
  int32_t run_cap;         /* longest register run of the diagonal walks before it
                              is recorded (bounds FP32 run sums): 0 = default
                              (128), else a power of two in [8, 1024] */
} lya_corr_opts;

typedef struct {
  double ref_pairs;        /* sum over forest pairs of len1*len2 (reference pair count) */
  double evaluated_pairs;  /* pixel pairs the kernel evaluated */
  double guard_rechecks;   /* pairs re-evaluated in FP64 inside the guard band */
  double runs_flushed;     /* register runs flushed into the shared histogram */
  double in_range_pairs;   /* pairs that landed in a bin */
  double kernel_ms;        /* device time of the last lya_corr_run pair kernel */
  double build_ms;         /* device time of the last lya_build_pairs */
  int64_t n_pairs;         /* forest pairs in the work queue */
  int32_t n_slots;
  int32_t n_forests;
  double guard_bound;      /* proven FP32 error bound, Mpc/h */
  double run_ms;           /* device time of the last lya_corr_run (all its work) */
  double run_ref_pairs;    /* reference pair count of the last run's slot range */
  int64_t launches;        /* kernels of this library launched by the context so far */
  double ref_pixels;       /* sum over forest pairs of len1+len2 */
  double adjoint_ms;       /* device time of the last lya_corr_adjoint's gradient kernels */
  double dist_mma_flops;   /* FP64 tensor-core flops of the last lya_dist_run (block products) */
} lya_stats_t;

/* ----------------------------------------------------------------- context */
int lya_ctx_create(int device, lya_ctx** out);
int lya_ctx_destroy(lya_ctx* ctx);
/* Message of the last failure on ctx (or of the last failure of this thread
 * when ctx is NULL). Never NULL. */
const char* lya_last_error(const lya_ctx* ctx);
int lya_version(void);

/* Histogram geometry; replaces the module constants rpmax, rtmax, numpix_rp,
 * numpix_rt (parameters.py:18-23) read by pair_correlation
 * (cuda_kernels.cpp:94-99).  np*nt <= 4096. */
int lya_set_bins(lya_ctx* ctx, double rpmax, double rtmax, int32_t np, int32_t nt);

/* Forest catalogue upload; replaces correlation_procedures_pycuda.init
 * (correlation_procedures_pycuda.py:16-111), which packs padded FP64 arrays and
 * copies them to the device.  Forests are given in forest.index order as CSR:
 * forest f owns pixels start[f]..start[f+1]-1 of dc, w, dw, z (and dl).
 * owner_slot[f] is the output histogram of pairs whose first forest is f (the
 * healpix pixel of forest_class.py:22-25, renumbered 0..n_slots-1) and must be
 * non-decreasing in f.  name[] identifies the quasar (same name: no pair).
 * dl, omega, odl2 may be NULL (needed by the distortion only). */
int lya_upload_forests(lya_ctx* ctx, int64_t n_forests, const int64_t* start, const double* dc, const double* w,
                       const double* dw, const double* z, const double* dl, const double* ux, const double* uy,
                       const double* uz, const double* ra, const double* dec, const int64_t* name,
                       const int32_t* owner_slot, int32_t n_slots, const double* omega, const double* odl2);

/* Catalogue upload from the deltas, with the projection done on the device:
 * replaces the per-quasar fill_dw(delta, loglam, project) of the ingest
 * (delta_reader.py:53, forest_class.py:48-68).  Arguments as
 * lya_upload_forests, with delta (per pixel) in place of dw and
 * log10(lambda) (loglam, per pixel) in place of dl; dw, the deltas' weighted
 * log-lambda offsets dl, omega = sum w and odl2 = sum w dl^2 are computed per
 * forest on the device (project = 1), or dw = delta w with dl, omega, odl2 = 0
 * (project = 0), exactly as fill_dw.  A forest whose weights sum to 0 is
 * LYA_ERR_DATA (numpy's average raises there). */
int lya_upload_deltas(lya_ctx* ctx, int64_t n_forests, const int64_t* start, const double* dc, const double* w,
                      const double* delta, const double* z, const double* loglam, const double* ux, const double* uy,
                      const double* uz, const double* ra, const double* dec, const int64_t* name,
                      const int32_t* owner_slot, int32_t n_slots, int32_t project);

/* The catalogue's dw, dl (per pixel, CSR order) and omega, odl2 (per forest)
 * as uploaded or as projected by lya_upload_deltas (host arrays; any may be
 * NULL).  The quasar attributes dw, delta_lambda, omega, omega_delta_lambda2
 * of forest_class.py:42-46. */
int lya_get_projection(lya_ctx* ctx, double* dw, double* dl, double* omega, double* odl2);

/* Neighbour lists on the device; replaces quasar.neighborhood
 * (forest_class.py:78-98) called per forest by two_point_per_pixel
 * (correlation_procedures_pycuda.py:144): f2 is a neighbour of f1 when
 * ((x1*x2 + y1*y2) + z1*z2) > mumin (mumin = cos(angmax) as numpy computes it),
 * name1 != name2 and ra1 < ra2.  The work queue holds every (f1, f2) pair,
 * grouped by f1.  *n_pairs_out receives the number of forest pairs. */
int lya_build_pairs(lya_ctx* ctx, double angmax, double mumin, int64_t* n_pairs_out);

/* Explicit work queue from the host, in place of lya_build_pairs: forest
 * pairs (f1[k], f2[k]) grouped by f1 (f1 non-decreasing). */
int lya_set_pairs(lya_ctx* ctx, int64_t n_pairs, const int32_t* f1, const int32_t* f2);

/* Keep only the work-queue pairs whose first forest's owner slot s has
 * keep[s] != 0 (keep: host array of n_slots flags); the queue stays grouped
 * by f1 and the reference pair counts of lya_stats follow.  Takes the place
 * of the reference's scatter of healpix pixels over MPI ranks
 * (2pla.py:87,102): a rank keeps the owner pixels assigned to it (any subset,
 * e.g. a cost-balanced one) and its runs bin only those. */
int lya_select_slots(lya_ctx* ctx, const uint8_t* keep);

/* Copy the current work queue to the host (n_pairs entries each). */
int lya_get_pairs(lya_ctx* ctx, int32_t* f1, int32_t* f2);

/* Per-slot pair histograms of the whole work queue in one persistent launch;
 * replaces the per-forest launch loop of two_point_per_pixel
 * (correlation_procedures_pycuda.py:141-166) and the pair_correlation kernel
 * (cuda_kernels.cpp:90-162).  Results stay on the device until lya_corr_get. */
int lya_corr_run(lya_ctx* ctx, const lya_corr_opts* opts);

/* Copy slots [slot_first, slot_first+n) to the host: hist[n][LYA_NQ][np*nt]
 * (FP64) and counts[n][np*nt] (pair counts).  Either pointer may be NULL. */
int lya_corr_get(lya_ctx* ctx, int32_t slot_first, int32_t n, double* hist, uint64_t* counts);

/* Gradient of L = sum_b g[b] * DW_b / W_b (totals over all slots of the last
 * lya_corr_run) with the pair bins held fixed: grad_dw and grad_w per pixel of
 * the catalogue (CSR order).  g has np*nt values; device_ptrs bit 0: grad_dw
 * and grad_w are device arrays on the context's device (else host arrays);
 * bit 1: g is a device array (else a host array).  lya_stats' adjoint_ms is
 * the device time of the gradient kernels.  No reference counterpart. */
int lya_corr_adjoint(lya_ctx* ctx, const double* g, double* grad_dw, double* grad_w, int32_t device_ptrs);

/* Totals over all owner slots of the last lya_corr_run: W[b] = sum w1w2 and
 * DW[b] = sum dw1dw2 (np*nt values each; host arrays, or device arrays when
 * device_ptrs is 1).  The sums post_processing.py:134-149 forms from the
 * per-pixel files; used for xi = DW/W without copying every pixel's
 * histograms.  No reference counterpart. */
int lya_corr_totals(lya_ctx* ctx, double* W, double* DW, int32_t device_ptrs);

/* Replace the weights w and weighted deltas dw of every pixel (CSR order, as
 * uploaded) without re-uploading the catalogue; host arrays, or device arrays
 * when device_ptrs is 1.  Used between forward evaluations of the adjoint
 * (fill_dw of forest_class.py:48-68 changes dw when delta or w change). */
int lya_update_weights(lya_ctx* ctx, const double* w, const double* dw, int32_t device_ptrs);

/* Distortion-matrix numerator D[np*nt][np*nt] and bin weights W[np*nt]
 * (FP64, host arrays, overwritten) summed over the work queue (build it with
 * lya_build_pairs, or pass the reference's subsampled neighbour lists with
 * lya_set_pairs); replaces distortion_per_pixel
 * (distortion_procedures_pycuda.py:195-279) and the kernels
 * precompute_distances, compute_etas, order_active, compute_d
 * (cuda_kernels.cpp:46-87, 165-278).  The normalised matrix of distortion.py:125
 * is D / W[:, None].  Needs dl, omega and odl2 at upload; a pixel whose
 * partners fall in more than 8 rt bins is reported as LYA_ERR_DATA. */
int lya_dist_run(lya_ctx* ctx, double* D, double* W);

/* Launch shape of lya_dist_run's kernel (0 = default: 512 threads per CTA,
 * rows staged 32 pixels at a time; 1..4 = 512/16, 512/24, 256/32, 256/16) and
 * an optional limit: max_items > 0 bins only the first max_items forest pairs
 * of the work queue (a timing sample for the autotuner), 0 = all.  Stays in
 * effect for later calls.  No reference counterpart. */
int lya_dist_config(lya_ctx* ctx, int32_t shape, int64_t max_items);

int lya_stats(lya_ctx* ctx, lya_stats_t* out);

/* Covariance of the per-pixel correlation estimates; replaces cov
 * (post_processing.py:30-52), fed by the reading loop of post_processing.py:
 * 134-149.  xi and w are host arrays [n_rows][np*nt] (xi = DW/W of an owner
 * pixel, 0 where W = 0, and w = W, in bin_coordinates order: bin p*nt + t,
 * post_processing.py:13-28); with xi and w both NULL the rows are the owner
 * slots of the last lya_corr_run, read on the device (n_rows is ignored).
 * Outputs (host, either may be NULL): mean[np*nt] (the weighted mean
 * correlation) and cov[np*nt][np*nt]; the covariance is also kept on the
 * device for lya_covariance_smooth.  A bin whose weights sum to 0 is
 * LYA_ERR_DATA (the reference's numba code raises ZeroDivisionError). */
int lya_covariance(lya_ctx* ctx, int64_t n_rows, const double* xi, const double* w, double* mean, double* cov);

/* Smoothed covariance; replaces cov_smooth (post_processing.py:54-91): the
 * correlation matrix averaged over pairs of bins with equal (|r_par step|,
 * |r_perp step|), scaled back by sqrt(C_aa C_bb).  cov is a host matrix
 * [np*nt][np*nt], or NULL for the one the last lya_covariance kept.  When a
 * variance is 0 the output is the unsmoothed covariance and *smoothed = 0, as
 * the reference returns it. */
int lya_covariance_smooth(lya_ctx* ctx, const double* cov, double* cov_smooth, int32_t* smoothed);

/* Histograms of one owner pixel without any device allocation.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory (device memory owned by another framework's caching allocator, a
 * fixed device-memory budget, allocation calls that must stay out of a
 * recorded sequence).  Every pointer is caller-owned device memory on
 * `device`: the catalogue as unpadded CSR (forest f owns pixels
 * start[f]..start[f+1]-1 of dc, w, dw, z), unit vectors ux, uy, uz per forest,
 * and the forest pairs (f1[k], f2[k]), all binned into one histogram;
 * outputs hist[LYA_NQ][np*nt] (FP64, same quantities as lya_corr_get) and
 * counts[np*nt], both overwritten.  Every pixel pair is evaluated with the
 * reference FP64 formula (the FP64 plain kernel).  The only scratch is a
 * file-scope device array of 4096 bins (320 KB per GPU that loads the
 * library, kept until exit): np*nt above 4096 is rejected with LYA_ERR_ARG.
 * The call makes `device` current itself (cudaSetDevice on the library's own,
 * statically linked, CUDA runtime).  The first call on a device does that
 * device's set-up (the array's device address, the kernels' shared-memory
 * limit, kernel loading, the SM count) and should come before any stream
 * capture; later calls make no set-up calls.  All calls share the array:
 * calls that overlap on the GPU race.  stream: a cudaStream_t, or NULL for the
 * default stream.  The call is asynchronous on that stream.
 * Preconditions the call does not check (it reads the caller's device memory
 * as given): start has n_forests+1 non-decreasing entries with start[0] = 0
 * and dc, w, dw, z hold start[n_forests] pixels; ux, uy, uz hold n_forests
 * entries; 0 <= f1[k], f2[k] < n_forests for k < n_pairs. */
int lya_corr_pixel_noalloc(int device, const double* dc, const double* w, const double* dw, const double* z,
                           const int64_t* start, const double* ux, const double* uy, const double* uz,
                           const int32_t* f1, const int32_t* f2, int64_t n_pairs, double rpmax, double rtmax,
                           int32_t np, int32_t nt, double* hist, uint64_t* counts, void* stream);

/* Test hooks for the failure paths (no counterpart in the reference).
 * lya_debug_fail_alloc: the device allocation made after `after` more
 * allocations of the library fails once (LYA_ERR_ALLOC from the call that
 * made it); -1 disarms.  LYA2PCF_FAIL_ALLOC=<after> in the environment arms it
 * when the library loads.  lya_debug_inject(ctx, 1): the next lya_corr_run's
 * pair kernel raises its device error flag, and the run returns
 * LYA_ERR_DEVICE as it does when the kernel finds a run record outside the
 * histogram.  Neither touches memory it should not: the context stays usable. */
int lya_debug_fail_alloc(int64_t after);
int lya_debug_inject(lya_ctx* ctx, int32_t what);

/* Shared-memory atomic throughput of `device` (no counterpart in the
 * reference): rates[0] FP64 atomicAdd at distinct addresses within a warp,
 * rates[1] FP64 atomicAdd into pseudo-random bins of a 2500-bin histogram,
 * rates[2] 32-bit integer atomicAdd at distinct addresses, in atomics per
 * second over the whole GPU (one-wave grid of 512-thread CTAs).  The
 * shared-atomic term of the pair kernel's roofline. */
int lya_probe_smem_atomics(int device, double* rates);

/* Device timer on the context's stream: op 0 records the start event, op 1
 * records the stop event, waits for it and writes the elapsed milliseconds. */
int lya_timer(lya_ctx* ctx, int32_t op, double* ms);

/* Block until all work queued on the context's stream has finished. */
int lya_sync(lya_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* LYA2PCF_H */
