// Internal declarations of the lya2pcf B200 library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "lya2pcf.h"

#define LYA_MAX_BINS 4096
#define LYA_WARP 32
// Zero pixels before the first and after the last forest of the padded pixel
// arrays: the kernels' software pipelines read up to 34 pixels past either end
// of a forest without bounds checks (the values are never used).
#define LYA_MARGIN 64

// Per-forest flags (DevCatalog::sorted): dc non-decreasing; and, in addition,
// every dc finite and in [0, LYA_LEAN_DC_MAX), which the lean walk of the FP32
// kernel requires for its error bound.
#define LYA_SORTED 1
#define LYA_LEAN 2
#define LYA_LEAN_DC_MAX 1.0e6

// Device-side statistics slots (unsigned long long counters).
enum { ST_EVALUATED = 0, ST_RECHECK = 1, ST_RUNS = 2, ST_INRANGE = 3, ST_ERROR = 4, ST_N = 8 };

// Forest catalogue on the device.  Per-pixel arrays use a padded CSR: forest f
// owns pixels pstart[f] .. pstart[f]+len[f]-1, with pstart[f] a multiple of 4 so
// every forest starts on a 32-byte boundary of the FP64 arrays, and
// LYA_MARGIN zero pixels before the first and after the last forest.
struct DevCatalog {
  int64_t n = 0;          // forests
  int64_t npix = 0;       // real pixels
  int64_t npad = 0;       // padded pixel slots
  int32_t n_slots = 0;
  int64_t* pstart = nullptr;   // [n]
  int32_t* len = nullptr;      // [n]
  uint8_t* sorted = nullptr;   // [n] LYA_SORTED | LYA_LEAN flags
  int32_t* slot = nullptr;     // [n] owner histogram
  double* ux = nullptr;        // [n]
  double* uy = nullptr;
  double* uz = nullptr;
  double* ra = nullptr;
  double* dec = nullptr;
  long long* name = nullptr;
  double* omega = nullptr;
  double* odl2 = nullptr;
  // FP64 per pixel (padded)
  double* dc = nullptr;
  double* w = nullptr;
  double* dw = nullptr;
  double* z = nullptr;
  double* dl = nullptr;
  // packed FP64 per pixel (padded): (dc, w, dw, z)
  double4* pix8 = nullptr;
  // FP32 per pixel (padded): (dc_hi, dc_lo, w, dw) and z
  float4* pix4 = nullptr;
  float* z32 = nullptr;
  bool has_dl = false;
  bool has_moments = false;
  int64_t n_not_lean = 0;      // forests without the LYA_LEAN flag
  int64_t cap_n = 0;           // allocated forests of the per-forest arrays
  int64_t cap_npad = 0;        // allocated padded pixel slots of the per-pixel arrays
};

// Staging of an upload: the caller's unpadded CSR arrays on the device, packed
// into the DevCatalog by k_pack.  Kept between uploads (grown, never shrunk).
struct UploadStaging {
  double* dc = nullptr;
  double* w = nullptr;
  double* dw = nullptr;
  double* z = nullptr;
  double* dl = nullptr;
  int64_t* start = nullptr;
  unsigned long long* zero_w = nullptr;   // [1] forests whose weights sum to 0
  int64_t cap_npix = 0, cap_n = 0;
};

// Scratch of the device neighbour search, kept between builds (grown, never
// shrunk), so a build allocates nothing once sized.
struct NbrScratch {
  int32_t* band = nullptr;      // [cap_n] band of each forest, then the sorted bands
  int32_t* band2 = nullptr;     // [cap_n]
  int32_t* sidx = nullptr;      // [cap_n] forests in (band, ra) order
  int32_t* sidx2 = nullptr;     // [cap_n]
  double* sra = nullptr;        // [cap_n] their ra
  double* sra2 = nullptr;       // [cap_n]
  int64_t* bstart = nullptr;    // [cap_band + 1]
  long long* counts = nullptr;  // [cap_n + 1]
  long long* offsets = nullptr; // [cap_n + 1]
  int* flag = nullptr;          // [1] some ra outside [0, 2 pi)
  double* tot = nullptr;        // [2] sum len1*len2, sum len1+len2
  void* tmp = nullptr;          // cub sort / scan scratch
  size_t tmp_bytes = 0;
  int64_t cap_n = 0, cap_band = 0;
  long long* h_out = nullptr;   // pinned [4]: pair count, then tot as double bits
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // build timing, read lazily by lya_stats
  bool timing_pending = false;
};

struct WorkQueue {
  int64_t n_pairs = 0;
  int64_t cap = 0;             // allocated entries of f1 and f2 (reused by later queues)
  int32_t* f1 = nullptr;       // [n_pairs] grouped by f1 (non-decreasing)
  int32_t* f2 = nullptr;       // [n_pairs]
  double ref_pairs = 0.0;      // sum len1*len2
  double ref_pixels = 0.0;     // sum len1+len2
};

// Scratch, outputs and captured graph of lya_dist_run (kept between calls).
struct DistScratch {
  double* D = nullptr;                 // [nb][nb]
  double* W = nullptr;                 // [nb]
  double* col = nullptr;               // column scratch of every CTA
  double* mom = nullptr;               // moment scratch of every CTA
  unsigned long long* err = nullptr;   // [3]: span errors, work counter, item count
  int nb = 0, max_len = 0, grid = 0;
  cudaGraphExec_t graph = nullptr;     // clear + distortion kernel
  alignas(16) unsigned char key[512] = {};   // the kernel parameters it was captured with
};

// Scratch of lya_select_slots (kept between calls, grown, never shrunk).
struct SelectScratch {
  uint8_t* keep = nullptr;      // [keep_cap] slot keep flags
  long long* pos = nullptr;     // [cap + 1] item flags, then their exclusive scan
  int32_t* o1 = nullptr;        // [cap] compacted queue
  int32_t* o2 = nullptr;
  double* tot = nullptr;        // [2] reference pixel pairs and pixels of the kept items
  void* tmp = nullptr;          // cub scan scratch
  size_t tmp_bytes = 0;
  int64_t cap = 0;
  int32_t keep_cap = 0;
  double* h_out = nullptr;      // pinned [3]: kept count (as long long bits), tot
};

// Scratch of lya_corr_adjoint (kept between calls, grown, never shrunk).
struct AdjScratch {
  double* g = nullptr;          // [nb] g on the device
  double* coef = nullptr;       // [2][nb] g/W, -g xi/W
  double* gdw = nullptr;        // [npad] gradients, padded layout
  double* gw = nullptr;
  double* out = nullptr;        // [npix] unpadded copy for host outputs
  int64_t* start = nullptr;     // [n + 1] CSR offsets
  int nb = 0;
  int64_t n = 0, npad = 0, npix = 0;
};

struct lya_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // kernel timing
  cudaEvent_t ev2 = nullptr, ev3 = nullptr;   // whole-call timing
  cudaEvent_t tev0 = nullptr, tev1 = nullptr; // lya_timer
  int64_t launches = 0;
  std::string err;

  bool bins_set = false;
  double rpmax = 200.0, rtmax = 200.0;
  int32_t np = 50, nt = 50;

  DevCatalog cat;
  std::vector<int64_t> h_start;  // host copy of the CSR offsets (unpadded)
  std::vector<int64_t> h_pstart;
  std::vector<int32_t> h_slot;

  UploadStaging stg;

  WorkQueue wq;
  NbrScratch nbr;
  SelectScratch sel;
  AdjScratch adj;
  int cos_variant = 0;

  // correlation outputs: per slot, LYA_NQ quantities as (hi, lo) FP64 pairs,
  // and pair counts
  double* hist = nullptr;            // [n_slots][LYA_NQ][2][nb]
  unsigned long long* counts = nullptr;  // [n_slots][nb]
  int32_t hist_slots = 0, hist_nb = 0;
  bool have_result = false;
  double* get_tmp = nullptr;             // lya_corr_get's combined (hi + lo) sums, kept between calls
  int64_t get_tmp_cap = 0;

  unsigned long long* stats = nullptr;   // [ST_N]
  int64_t* cta_begin = nullptr;          // [max ctas + 1]
  int32_t cta_cap = 0;

  // persistent scratch of lya_corr_run, so a run allocates nothing once sized
  // and its stream work can be captured in a CUDA graph and replayed
  long long* cost = nullptr;             // [cost_cap] per-item cost, then its prefix sum
  int64_t cost_cap = 0;
  void* scan_tmp = nullptr;              // cub scan scratch
  size_t scan_tmp_bytes = 0;
  unsigned long long* h_stats = nullptr; // pinned host copy: [ST_N] counters + range pair count (as double bits)
  cudaGraphExec_t run_graph = nullptr;   // the last run, captured
  alignas(16) unsigned char run_graph_key[512] = {};   // what it was captured for (see corr.cu)
  int64_t graph_launches = 0;            // runs replayed from the captured graph

  lya_stats_t last{};
  bool inject_device_error = false;      // test hook: the next run's pair kernel raises its error flag

  DistScratch dist;
  int32_t dist_shape = 0;                // lya_dist_config: launch shape of the distortion kernel
  int64_t dist_max_items = 0;            // lya_dist_config: 0 = every forest pair, else the first n

  // covariance post-processing: the last covariance, kept for lya_covariance_smooth
  double* cov = nullptr;                 // [cov_nb][cov_nb]
  int32_t cov_nb = 0;
  bool have_cov = false;
};

// ------------------------------------------------------------------ errors
int lya_fail(lya_ctx* ctx, int code, const char* fmt, ...);

#define LYA_CHECK_CUDA(ctx, call)                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return lya_fail((ctx), LYA_ERR_CUDA, "%s failed: %s", #call,   \
                                           cudaGetErrorString(e_));                         \
  } while (0)

// Allocation-failure hook (lya_debug_fail_alloc, or LYA2PCF_FAIL_ALLOC in the
// environment): true when this device allocation is the one to fail.
bool lya_alloc_fault();

template <typename T>
inline cudaError_t lya_alloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  if (lya_alloc_fault()) return cudaErrorMemoryAllocation;
  return cudaMalloc((void**)p, count * sizeof(T));
}

template <typename T>
inline void lya_free(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void lya_free_catalog(DevCatalog& c);
void lya_free_queue(WorkQueue& q);
void lya_free_nbr_scratch(NbrScratch& s);
// build_ms of the last neighbour build, once its stop event has completed
void lya_resolve_build_timing(lya_ctx* ctx);
// Room for n pairs in q (f1, f2), keeping the buffers when they are large
// enough; n_pairs is left to the caller.
cudaError_t lya_queue_reserve(WorkQueue& q, int64_t n);

// ------------------------------------------------------------------ device math
// cos of the angle between two lines of sight, FP64, in the contraction order
// nvcc gives the reference's "x1*x2 + y1*y2 + z1*z2" (cuda_kernels.cpp:131);
// variant selects the order (see the oracle's orc_cos12 for the list).
__device__ __forceinline__ double lya_cos12(double x1, double y1, double z1, double x2, double y2, double z2,
                                             int variant) {
  if (variant == 0) return __fma_rn(z1, z2, __fma_rn(x1, x2, __dmul_rn(y1, y2)));
  if (variant == 1) return __fma_rn(z1, z2, __fma_rn(y1, y2, __dmul_rn(x1, x2)));
  return __dadd_rn(__dadd_rn(__dmul_rn(x1, x2), __dmul_rn(y1, y2)), __dmul_rn(z1, z2));
}

// D(8x8) += A(8x4) B(4x8) in FP64 on the tensor cores, one warp (FP64 has no
// tcgen05 kind).  Fragments: a = A[lane/4][lane%4], b = B[lane%4][lane/4],
// d = D[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void lya_dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// FP64 tensor-core MMA, D (16x8) += A (16x8, row-major) x B (8x8, column-major).
// Fragments, with g = lane / 4 and q = lane % 4: a0 (g, q), a1 (g+8, q),
// a2 (g, q+4), a3 (g+8, q+4); b0 (q, g), b1 (q+4, g); c0, c1 (g, 2q and 2q+1),
// c2, c3 (g+8, 2q and 2q+1).  Four times the work of one m8n8k4 per instruction.
__device__ __forceinline__ void lya_dmma_16x8x8(double (&c)[4], double a0, double a1, double a2, double a3,
                                                double b0, double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
               "{%0, %1, %2, %3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// ------------------------------------------------------------------ launchers
int lya_corr_launch(lya_ctx* ctx, const lya_corr_opts* o);
int lya_build_queue(lya_ctx* ctx, double angmax, double mumin);
int lya_adjoint_launch(lya_ctx* ctx, const double* g, double* grad_dw, double* grad_w, int device_ptrs);

