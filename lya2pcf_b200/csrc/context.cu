// Context, catalogue upload and result copy-out of the lya2pcf B200 library.
//
// The upload replaces correlation_procedures_pycuda.init
// (correlation_procedures_pycuda.py:16-111): instead of host-packed
// [n_forest x max_lenght] padded FP64 arrays, the caller's unpadded CSR arrays
// are copied once and packed on the device into
//   * FP64 per-pixel arrays (dc, w, dw, z, dl) on a 4-pixel-aligned CSR, read by
//     the FP64 kernels and by the FP32 kernel's guard-band recheck;
//   * an FP32 float4 per pixel (dc_hi, dc_lo, w, dw) plus FP32 z, read by the
//     FP32 kernel: dc = dc_hi + dc_lo to ~2^-48 relative, so FP32 differences
//     of comoving distances stay accurate to ~1e-5 Mpc/h.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "lya_internal.cuh"

static thread_local std::string g_thread_err;

// ------------------------------------------------------------------ test hooks
// Allocation-failure hook: the device allocation made after `g_fail_alloc_in`
// more allocations fails once with cudaErrorMemoryAllocation (-1 = never).
// LYA2PCF_FAIL_ALLOC=<n> in the environment arms it when the library loads.
static std::atomic<long long> g_fail_alloc_in{[] {
  const char* v = getenv("LYA2PCF_FAIL_ALLOC");
  return v && *v ? atoll(v) : -1ll;
}()};

bool lya_alloc_fault() {
  long long n = g_fail_alloc_in.load();
  while (n >= 0) {
    if (g_fail_alloc_in.compare_exchange_weak(n, n - 1)) return n == 0;
  }
  return false;
}

extern "C" int lya_debug_fail_alloc(int64_t after) {
  g_fail_alloc_in.store(after < 0 ? -1 : (long long)after);
  return LYA_OK;
}

extern "C" int lya_debug_inject(lya_ctx* ctx, int32_t what) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_debug_inject: ctx is NULL");
  if (what != 1) return lya_fail(ctx, LYA_ERR_ARG, "lya_debug_inject: unknown hook %d", what);
  ctx->inject_device_error = true;
  return LYA_OK;
}

int lya_fail(lya_ctx* ctx, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_thread_err = buf;
  if (ctx) ctx->err = buf;
  return code;
}

void lya_free_catalog(DevCatalog& c) {
  lya_free(c.pstart); lya_free(c.len); lya_free(c.sorted); lya_free(c.slot);
  lya_free(c.ux); lya_free(c.uy); lya_free(c.uz); lya_free(c.ra); lya_free(c.dec); lya_free(c.name);
  lya_free(c.omega); lya_free(c.odl2);
  lya_free(c.dc); lya_free(c.w); lya_free(c.dw); lya_free(c.z); lya_free(c.dl);
  lya_free(c.pix4); lya_free(c.z32); lya_free(c.pix8);
  c = DevCatalog{};
}

void lya_free_queue(WorkQueue& q) {
  lya_free(q.f1); lya_free(q.f2);
  q = WorkQueue{};
}

static void free_staging(UploadStaging& t) {
  lya_free(t.dc); lya_free(t.w); lya_free(t.dw); lya_free(t.z); lya_free(t.dl); lya_free(t.start);
  lya_free(t.zero_w);
  t = UploadStaging{};
}

void lya_free_nbr_scratch(NbrScratch& s) {
  lya_free(s.band); lya_free(s.band2); lya_free(s.sidx); lya_free(s.sidx2); lya_free(s.sra); lya_free(s.sra2);
  lya_free(s.bstart); lya_free(s.counts); lya_free(s.offsets); lya_free(s.flag); lya_free(s.tot);
  if (s.tmp) cudaFree(s.tmp);
  if (s.h_out) cudaFreeHost(s.h_out);
  if (s.ev0) cudaEventDestroy(s.ev0);
  if (s.ev1) cudaEventDestroy(s.ev1);
  s = NbrScratch{};
}

// Device arrays of a catalogue of n forests and npad padded pixel slots.  The
// arrays of the previous upload are kept when they are large enough, so that
// uploading a catalogue of the same size again allocates and frees nothing
// (and the buffers a captured run reads keep their addresses).
static cudaError_t catalog_reserve(DevCatalog& c, int64_t n, int64_t npad) {
  if (c.pstart && n <= c.cap_n && npad <= c.cap_npad) return cudaSuccess;
  lya_free_catalog(c);
  cudaError_t e = cudaSuccess;
#define ALLOC(p, cnt) if (e == cudaSuccess) e = lya_alloc(&(p), (size_t)(cnt))
  ALLOC(c.pstart, n); ALLOC(c.len, n); ALLOC(c.sorted, n); ALLOC(c.slot, n);
  ALLOC(c.ux, n); ALLOC(c.uy, n); ALLOC(c.uz, n); ALLOC(c.ra, n); ALLOC(c.dec, n); ALLOC(c.name, n);
  ALLOC(c.omega, n); ALLOC(c.odl2, n);
  ALLOC(c.dc, npad); ALLOC(c.w, npad); ALLOC(c.dw, npad); ALLOC(c.z, npad); ALLOC(c.dl, npad);
  ALLOC(c.pix4, npad); ALLOC(c.z32, npad); ALLOC(c.pix8, npad);
#undef ALLOC
  if (e != cudaSuccess) {
    lya_free_catalog(c);
    return e;
  }
  c.cap_n = n;
  c.cap_npad = npad;
  return cudaSuccess;
}

// Staging arrays for an upload of n forests and npix pixels (kept between uploads).
static cudaError_t staging_reserve(UploadStaging& t, int64_t n, int64_t npix) {
  if (t.start && n <= t.cap_n && npix <= t.cap_npix) return cudaSuccess;
  free_staging(t);
  cudaError_t e = cudaSuccess;
#define ALLOC(p, cnt) if (e == cudaSuccess) e = lya_alloc(&(p), (size_t)(cnt))
  ALLOC(t.dc, npix); ALLOC(t.w, npix); ALLOC(t.dw, npix); ALLOC(t.z, npix); ALLOC(t.dl, npix);
  ALLOC(t.start, n + 1); ALLOC(t.zero_w, 1);
#undef ALLOC
  if (e != cudaSuccess) {
    free_staging(t);
    return e;
  }
  t.cap_n = n;
  t.cap_npix = npix;
  return cudaSuccess;
}

cudaError_t lya_queue_reserve(WorkQueue& q, int64_t n) {
  if (n <= q.cap && q.f1 && q.f2) return cudaSuccess;
  lya_free_queue(q);
  cudaError_t e = lya_alloc(&q.f1, (size_t)std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = lya_alloc(&q.f2, (size_t)std::max<int64_t>(n, 1));
  if (e != cudaSuccess) { lya_free_queue(q); return e; }
  q.cap = std::max<int64_t>(n, 1);
  return cudaSuccess;
}

extern "C" int lya_version(void) { return 10000; }

extern "C" const char* lya_last_error(const lya_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  return g_thread_err.c_str();
}

extern "C" int lya_ctx_create(int device, lya_ctx** out) {
  if (!out) return lya_fail(nullptr, LYA_ERR_ARG, "lya_ctx_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return lya_fail(nullptr, LYA_ERR_CUDA, "lya_ctx_create: no CUDA device (%s)", cudaGetErrorString(e));
  if (device < 0 || device >= ndev)
    return lya_fail(nullptr, LYA_ERR_ARG, "lya_ctx_create: device %d out of range [0,%d)", device, ndev);
  lya_ctx* ctx = new (std::nothrow) lya_ctx();
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ALLOC, "lya_ctx_create: host allocation failed");
  ctx->device = device;
  int rc = LYA_OK;
  do {
    if ((e = cudaSetDevice(device)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
      rc = LYA_ERR_CUDA; break;
    }
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->ev2)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->ev3)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->tev0)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = cudaEventCreate(&ctx->tev1)) != cudaSuccess) { rc = LYA_ERR_CUDA; break; }
    if ((e = lya_alloc(&ctx->stats, ST_N)) != cudaSuccess) { rc = LYA_ERR_ALLOC; break; }
    if ((e = cudaMallocHost((void**)&ctx->h_stats, sizeof(unsigned long long) * (ST_N + 1))) != cudaSuccess) {
      rc = LYA_ERR_ALLOC; break;
    }
  } while (0);
  if (rc != LYA_OK) {
    lya_fail(nullptr, rc, "lya_ctx_create: %s", cudaGetErrorString(e));
    lya_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return LYA_OK;
}

extern "C" int lya_ctx_destroy(lya_ctx* ctx) {
  if (!ctx) return LYA_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  lya_free_catalog(ctx->cat);
  free_staging(ctx->stg);
  lya_free_queue(ctx->wq);
  lya_free_nbr_scratch(ctx->nbr);
  lya_free(ctx->sel.keep); lya_free(ctx->sel.pos); lya_free(ctx->sel.o1); lya_free(ctx->sel.o2);
  lya_free(ctx->sel.tot);
  if (ctx->sel.tmp) cudaFree(ctx->sel.tmp);
  if (ctx->sel.h_out) cudaFreeHost(ctx->sel.h_out);
  lya_free(ctx->get_tmp);
  lya_free(ctx->adj.g); lya_free(ctx->adj.coef); lya_free(ctx->adj.gdw); lya_free(ctx->adj.gw);
  lya_free(ctx->adj.out); lya_free(ctx->adj.start);
  lya_free(ctx->hist); lya_free(ctx->counts); lya_free(ctx->stats); lya_free(ctx->cta_begin);
  lya_free(ctx->cost);
  lya_free(ctx->cov);
  lya_free(ctx->dist.D); lya_free(ctx->dist.W); lya_free(ctx->dist.col); lya_free(ctx->dist.mom);
  lya_free(ctx->dist.err);
  if (ctx->dist.graph) cudaGraphExecDestroy(ctx->dist.graph);
  if (ctx->scan_tmp) cudaFree(ctx->scan_tmp);
  if (ctx->h_stats) cudaFreeHost(ctx->h_stats);
  if (ctx->run_graph) cudaGraphExecDestroy(ctx->run_graph);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev2) cudaEventDestroy(ctx->ev2);
  if (ctx->ev3) cudaEventDestroy(ctx->ev3);
  if (ctx->tev0) cudaEventDestroy(ctx->tev0);
  if (ctx->tev1) cudaEventDestroy(ctx->tev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LYA_OK;
}

extern "C" int lya_set_bins(lya_ctx* ctx, double rpmax, double rtmax, int32_t np, int32_t nt) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_set_bins: ctx is NULL");
  if (!(rpmax > 0) || !(rtmax > 0) || np <= 0 || nt <= 0 || (int64_t)np * nt > LYA_MAX_BINS)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_set_bins: need rpmax, rtmax > 0 and 0 < np*nt <= %d (got %g %g %d %d)",
                    LYA_MAX_BINS, rpmax, rtmax, np, nt);
  ctx->rpmax = rpmax; ctx->rtmax = rtmax; ctx->np = np; ctx->nt = nt;
  ctx->bins_set = true;
  ctx->have_result = false;
  return LYA_OK;
}

// ------------------------------------------------------------------ packing
__global__ void k_pack(int64_t n, const int64_t* __restrict__ start, const int64_t* __restrict__ pstart,
                       const double* __restrict__ dc, const double* __restrict__ w, const double* __restrict__ dw,
                       const double* __restrict__ z, const double* __restrict__ dl, double* __restrict__ o_dc,
                       double* __restrict__ o_w, double* __restrict__ o_dw, double* __restrict__ o_z,
                       double* __restrict__ o_dl, double4* __restrict__ o_pix8, float4* __restrict__ o_pix4,
                       float* __restrict__ o_z32,
                       int32_t* __restrict__ o_len, uint8_t* __restrict__ o_sorted) {
  for (int64_t f = blockIdx.x; f < n; f += gridDim.x) {
    const int64_t s = start[f], L = start[f + 1] - s, d = pstart[f];
    int ok = 1, lean = 1;
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) {
      const double x = dc[s + k];
      // the FP32 error bound of the lean walk assumes 0 <= dc < 1e6 Mpc/h
      if (!(x >= 0.0 && x < LYA_LEAN_DC_MAX)) lean = 0;
      o_dc[d + k] = x;
      o_w[d + k] = w[s + k];
      o_dw[d + k] = dw[s + k];
      o_z[d + k] = z[s + k];
      if (dl) o_dl[d + k] = dl[s + k];
      o_pix8[d + k] = make_double4(x, w[s + k], dw[s + k], z[s + k]);
      const float hi = __double2float_rn(x);
      const float lo = __double2float_rn(x - (double)hi);
      o_pix4[d + k] = make_float4(hi, lo, __double2float_rn(w[s + k]), __double2float_rn(dw[s + k]));
      o_z32[d + k] = __double2float_rn(z[s + k]);
      if (k + 1 < L && !(x <= dc[s + k + 1])) ok = 0;
    }
    ok = __syncthreads_and(ok);
    lean = __syncthreads_and(lean);
    if (threadIdx.x == 0) {
      o_len[f] = (int32_t)L;
      o_sorted[f] = (uint8_t)(ok ? (lean ? (LYA_SORTED | LYA_LEAN) : LYA_SORTED) : 0);
    }
    __syncthreads();
  }
}

// Device projection of the deltas, quasar.fill_dw (forest_class.py:48-68), one
// block per forest: on entry dw holds delta and dl holds log10(lambda); on exit
// dw = w (delta - <delta> - dl <dl delta>/<dl^2>), dl = loglam - <loglam>, and
// omega = sum w, odl2 = sum dl^2 w (<.> weighted by w, in the reference's
// operation order; <dl^2> = 0, e.g. a one-pixel forest, gives NaN as numpy
// does).  project = 0: dw = delta w, dl = omega = odl2 = 0.  A forest whose
// weights sum to 0 is counted in zero_w (numpy's average raises there).
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < nw; ++k) t += red[k];
  return t;
}

__global__ void k_project(int64_t n, const int64_t* __restrict__ start, const double* __restrict__ w,
                          double* __restrict__ dw, double* __restrict__ dl, double* __restrict__ omega,
                          double* __restrict__ odl2, int project, unsigned long long* __restrict__ zero_w) {
  __shared__ double red[32];
  for (int64_t f = blockIdx.x; f < n; f += gridDim.x) {
    const int64_t a = start[f], L = start[f + 1] - a;
    if (!project) {
      for (int64_t k = threadIdx.x; k < L; k += blockDim.x) { dw[a + k] = dw[a + k] * w[a + k]; dl[a + k] = 0.0; }
      if (threadIdx.x == 0) { omega[f] = 0.0; odl2[f] = 0.0; }
      continue;
    }
    double sw = 0.0, swd = 0.0, swl = 0.0;
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) {
      const double wk = w[a + k];
      sw += wk;
      swd += dw[a + k] * wk;
      swl += dl[a + k] * wk;
    }
    sw = block_sum(sw, red);
    swd = block_sum(swd, red);
    swl = block_sum(swl, red);
    if (L > 0 && sw == 0.0 && threadIdx.x == 0) atomicAdd(zero_w, 1ull);
    const double deltaprom = swd / sw, lam = swl / sw;
    double s2 = 0.0, sld = 0.0;
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) {
      const double wk = w[a + k], x = dl[a + k] - lam;
      s2 += x * x * wk;
      sld += x * dw[a + k] * wk;
    }
    s2 = block_sum(s2, red);
    sld = block_sum(sld, red);
    const double ldprom = sld / sw, llprom = s2 / sw;
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) {
      const double wk = w[a + k], x = dl[a + k] - lam;
      dw[a + k] = wk * ((dw[a + k] - deltaprom) - x * ldprom / llprom);
      dl[a + k] = x;
    }
    if (threadIdx.x == 0) { omega[f] = sw; odl2[f] = s2; }
    __syncthreads();
  }
}

// ingest: -1 = forests with dw, dl, omega, odl2 given; 0 or 1 = deltas and
// log-lambda given in dw and dl, projected on the device (1) or not (0).
static int upload_impl(lya_ctx* ctx, int64_t n, const int64_t* start, const double* dc, const double* w,
                       const double* dw, const double* z, const double* dl, const double* ux, const double* uy,
                       const double* uz, const double* ra, const double* dec, const int64_t* name,
                       const int32_t* owner_slot, int32_t n_slots, const double* omega, const double* odl2,
                       int ingest) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_upload_forests: ctx is NULL");
  if (n < 0 || n >= (int64_t)INT32_MAX) return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: bad n_forests %lld",
                                                       (long long)n);
  if (!start || (n > 0 && (!ux || !uy || !uz || !ra || !dec || !name || !owner_slot)))
    return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: required pointer is NULL");
  if (n_slots < 0 || (n > 0 && n_slots == 0)) return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: bad n_slots");
  if (start[0] != 0) return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: start[0] must be 0");
  for (int64_t f = 0; f < n; ++f) {
    if (start[f + 1] < start[f]) return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: start not non-decreasing at %lld",
                                                 (long long)f);
    if (start[f + 1] - start[f] > 65536)
      return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: forest %lld longer than 65536 pixels", (long long)f);
    if (owner_slot[f] < 0 || owner_slot[f] >= n_slots)
      return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: owner_slot[%lld]=%d outside [0,%d)", (long long)f,
                      owner_slot[f], n_slots);
    if (f > 0 && owner_slot[f] < owner_slot[f - 1])
      return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: owner_slot must be non-decreasing (forest %lld)",
                      (long long)f);
  }
  const int64_t npix = start[n];
  if (npix > 0 && (!dc || !w || !dw || !z)) return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_forests: pixel array NULL");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->wq.n_pairs = 0;   // the queue's buffers are kept for the next build
  ctx->have_result = false;

  ctx->h_start.assign(start, start + n + 1);
  ctx->h_slot.assign(owner_slot, owner_slot + n);
  ctx->h_pstart.resize(n);
  int64_t off = LYA_MARGIN;
  for (int64_t f = 0; f < n; ++f) {
    ctx->h_pstart[f] = off;
    off += ((start[f + 1] - start[f]) + 3) & ~int64_t(3);
  }
  const int64_t npad = off + LYA_MARGIN;
  cudaError_t e = catalog_reserve(ctx->cat, n, npad);
  if (e == cudaSuccess) e = staging_reserve(ctx->stg, n, npix);
  if (e != cudaSuccess) {
    lya_free_catalog(ctx->cat);
    free_staging(ctx->stg);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_upload_forests: device allocation failed (%s)", cudaGetErrorString(e));
  }
  DevCatalog& c = ctx->cat;
  c.n = n; c.npix = npix; c.npad = npad; c.n_slots = n_slots;
  c.has_dl = dl != nullptr;
  c.has_moments = (omega != nullptr && odl2 != nullptr) || ingest >= 0;
  c.n_not_lean = 0;
  double *t_dc = ctx->stg.dc, *t_w = ctx->stg.w, *t_dw = ctx->stg.dw, *t_z = ctx->stg.z;
  double* t_dl = dl ? ctx->stg.dl : nullptr;
  int64_t* t_start = ctx->stg.start;
  cudaStream_t s = ctx->stream;
  auto H2D = [&](void* d, const void* h, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
  };
  H2D(c.pstart, ctx->h_pstart.data(), sizeof(int64_t) * n);
  H2D(c.slot, owner_slot, sizeof(int32_t) * n);
  H2D(c.ux, ux, sizeof(double) * n); H2D(c.uy, uy, sizeof(double) * n); H2D(c.uz, uz, sizeof(double) * n);
  H2D(c.ra, ra, sizeof(double) * n); H2D(c.dec, dec, sizeof(double) * n);
  H2D(c.name, name, sizeof(int64_t) * n);
  if (omega) H2D(c.omega, omega, sizeof(double) * n);
  if (odl2) H2D(c.odl2, odl2, sizeof(double) * n);
  H2D(t_start, start, sizeof(int64_t) * (n + 1));
  H2D(t_dc, dc, sizeof(double) * npix); H2D(t_w, w, sizeof(double) * npix); H2D(t_dw, dw, sizeof(double) * npix);
  H2D(t_z, z, sizeof(double) * npix);
  if (dl) H2D(t_dl, dl, sizeof(double) * npix);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.dc, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.w, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.dw, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.z, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.dl, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.pix4, 0, sizeof(float4) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.z32, 0, sizeof(float) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.pix8, 0, sizeof(double4) * npad, s);
  if (e == cudaSuccess && !omega) e = cudaMemsetAsync(c.omega, 0, sizeof(double) * n, s);
  if (e == cudaSuccess && !odl2) e = cudaMemsetAsync(c.odl2, 0, sizeof(double) * n, s);
  unsigned long long* zero_w = nullptr;
  if (e == cudaSuccess && ingest >= 0 && n > 0) {
    zero_w = ctx->stg.zero_w;
    e = cudaMemsetAsync(zero_w, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
      const int blocks = (int)std::min<int64_t>(n, (int64_t)ctx->num_sms * 16);
      k_project<<<blocks, 128, 0, s>>>(n, t_start, t_w, t_dw, t_dl, c.omega, c.odl2, ingest, zero_w);
      ctx->launches++;
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess && n > 0) {
    int blocks = (int)std::min<int64_t>(n, (int64_t)ctx->num_sms * 16);
    k_pack<<<blocks, 128, 0, s>>>(n, t_start, c.pstart, t_dc, t_w, t_dw, t_z, t_dl, c.dc, c.w, c.dw, c.z, c.dl,
                                  c.pix8, c.pix4, c.z32, c.len, c.sorted);
    ctx->launches++;
    e = cudaGetLastError();
  }
  // forests the FP32 kernel's lean walk cannot take (they need the second pass)
  std::vector<uint8_t> flags((size_t)n);
  unsigned long long nzero = 0;
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(flags.data(), c.sorted, (size_t)n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && zero_w) e = cudaMemcpyAsync(&nzero, zero_w, sizeof(nzero), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && nzero) {
    lya_free_catalog(ctx->cat);
    return lya_fail(ctx, LYA_ERR_DATA, "lya_upload_deltas: %llu forests have weights summing to 0", nzero);
  }
  if (e != cudaSuccess) {
    lya_free_catalog(ctx->cat);
    return lya_fail(ctx, LYA_ERR_CUDA, "lya_upload_forests: %s", cudaGetErrorString(e));
  }
  c.n_not_lean = 0;
  for (int64_t f = 0; f < n; ++f) c.n_not_lean += (flags[f] & LYA_LEAN) ? 0 : 1;
  return LYA_OK;
}

extern "C" int lya_upload_forests(lya_ctx* ctx, int64_t n, const int64_t* start, const double* dc, const double* w,
                                  const double* dw, const double* z, const double* dl, const double* ux,
                                  const double* uy, const double* uz, const double* ra, const double* dec,
                                  const int64_t* name, const int32_t* owner_slot, int32_t n_slots,
                                  const double* omega, const double* odl2) {
  return upload_impl(ctx, n, start, dc, w, dw, z, dl, ux, uy, uz, ra, dec, name, owner_slot, n_slots, omega, odl2,
                     -1);
}

extern "C" int lya_upload_deltas(lya_ctx* ctx, int64_t n, const int64_t* start, const double* dc, const double* w,
                                 const double* delta, const double* z, const double* loglam, const double* ux,
                                 const double* uy, const double* uz, const double* ra, const double* dec,
                                 const int64_t* name, const int32_t* owner_slot, int32_t n_slots, int32_t project) {
  if (ctx && start && n > 0 && start[n] > 0 && !loglam)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_upload_deltas: loglam is NULL");
  return upload_impl(ctx, n, start, dc, w, delta, z, loglam, ux, uy, uz, ra, dec, name, owner_slot, n_slots, nullptr,
                     nullptr, project ? 1 : 0);
}

extern "C" int lya_get_projection(lya_ctx* ctx, double* dw, double* dl, double* omega, double* odl2) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_get_projection: ctx is NULL");
  const DevCatalog& c = ctx->cat;
  if (c.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_get_projection: no forests uploaded");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  std::vector<double> pad((size_t)c.npad);
  for (int k = 0; k < 2; ++k) {
    double* out = k == 0 ? dw : dl;
    if (!out) continue;
    LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(pad.data(), k == 0 ? c.dw : c.dl, sizeof(double) * c.npad,
                                        cudaMemcpyDeviceToHost, s));
    LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    for (int64_t f = 0; f < c.n; ++f) {
      const int64_t a = ctx->h_start[f], L = ctx->h_start[f + 1] - a;
      std::copy(pad.begin() + ctx->h_pstart[f], pad.begin() + ctx->h_pstart[f] + L, out + a);
    }
  }
  if (omega) LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(omega, c.omega, sizeof(double) * c.n, cudaMemcpyDeviceToHost, s));
  if (odl2) LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(odl2, c.odl2, sizeof(double) * c.n, cudaMemcpyDeviceToHost, s));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  return LYA_OK;
}

// ------------------------------------------------------------------ weights update
__global__ void k_repack_weights(int64_t n, const int64_t* __restrict__ start, const int64_t* __restrict__ pstart,
                                 const double* __restrict__ w, const double* __restrict__ dw,
                                 double* __restrict__ o_w, double* __restrict__ o_dw, double4* __restrict__ o_pix8,
                                 float4* __restrict__ o_pix4) {
  for (int64_t f = blockIdx.x; f < n; f += gridDim.x) {
    const int64_t s = start[f], L = start[f + 1] - s, d = pstart[f];
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) {
      const double wv = w[s + k], dv = dw[s + k];
      o_w[d + k] = wv;
      o_dw[d + k] = dv;
      o_pix8[d + k].y = wv;
      o_pix8[d + k].z = dv;
      o_pix4[d + k].z = __double2float_rn(wv);
      o_pix4[d + k].w = __double2float_rn(dv);
    }
  }
}

extern "C" int lya_update_weights(lya_ctx* ctx, const double* w, const double* dw, int32_t device_ptrs) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_update_weights: ctx is NULL");
  if (ctx->cat.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_update_weights: no forests uploaded");
  const int64_t npix = ctx->cat.npix, n = ctx->cat.n;
  if (npix > 0 && (!w || !dw)) return lya_fail(ctx, LYA_ERR_ARG, "lya_update_weights: NULL array");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  double *tw = nullptr, *tdw = nullptr;
  int64_t* ts = nullptr;
  cudaError_t e = lya_alloc(&ts, n + 1);
  if (e == cudaSuccess && !device_ptrs) e = lya_alloc(&tw, npix);
  if (e == cudaSuccess && !device_ptrs) e = lya_alloc(&tdw, npix);
  if (e != cudaSuccess) {
    lya_free(ts); lya_free(tw); lya_free(tdw);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_update_weights: allocation failed");
  }
  const double* sw = device_ptrs ? w : tw;
  const double* sdw = device_ptrs ? dw : tdw;
  e = cudaMemcpyAsync(ts, ctx->h_start.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !device_ptrs) e = cudaMemcpyAsync(tw, w, sizeof(double) * npix, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !device_ptrs) e = cudaMemcpyAsync(tdw, dw, sizeof(double) * npix, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<int64_t>(n, (int64_t)ctx->num_sms * 16);
    k_repack_weights<<<blocks, 128, 0, s>>>(n, ts, ctx->cat.pstart, sw, sdw, ctx->cat.w, ctx->cat.dw, ctx->cat.pix8,
                                            ctx->cat.pix4);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  lya_free(ts); lya_free(tw); lya_free(tdw);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_update_weights: %s", cudaGetErrorString(e));
  ctx->have_result = false;
  return LYA_OK;
}

// ------------------------------------------------------------------ work queue from the host
__global__ void k_check_pairs(int64_t np, const int32_t* f1, const int32_t* f2, int64_t n, unsigned long long* err) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < np; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = f1[k], b = f2[k];
    if (a < 0 || a >= n || b < 0 || b >= n || (k > 0 && f1[k - 1] > a)) atomicAdd(err, 1ull);
  }
}

extern "C" int lya_set_pairs(lya_ctx* ctx, int64_t n_pairs, const int32_t* f1, const int32_t* f2) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_set_pairs: ctx is NULL");
  if (n_pairs < 0 || (n_pairs > 0 && (!f1 || !f2))) return lya_fail(ctx, LYA_ERR_ARG, "lya_set_pairs: bad arguments");
  if (ctx->cat.n == 0 && n_pairs > 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_set_pairs: upload forests first");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->have_result = false;
  WorkQueue& q = ctx->wq;
  q.n_pairs = 0;
  cudaError_t e = lya_queue_reserve(q, n_pairs);
  if (e != cudaSuccess) {
    lya_free_queue(q);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_set_pairs: device allocation failed");
  }
  double ref = 0.0, refpix = 0.0;
  for (int64_t k = 0; k < n_pairs; ++k) {
    if (f1[k] < 0 || f1[k] >= ctx->cat.n || f2[k] < 0 || f2[k] >= ctx->cat.n) {
      lya_free_queue(q);
      return lya_fail(ctx, LYA_ERR_ARG, "lya_set_pairs: pair %lld references a forest outside [0,%lld)", (long long)k,
                      (long long)ctx->cat.n);
    }
    if (k > 0 && f1[k] < f1[k - 1]) {
      lya_free_queue(q);
      return lya_fail(ctx, LYA_ERR_ARG, "lya_set_pairs: f1 must be non-decreasing (pair %lld)", (long long)k);
    }
    const double l1 = (double)(ctx->h_start[f1[k] + 1] - ctx->h_start[f1[k]]);
    const double l2 = (double)(ctx->h_start[f2[k] + 1] - ctx->h_start[f2[k]]);
    ref += l1 * l2;
    refpix += l1 + l2;
  }
  q.n_pairs = n_pairs;
  q.ref_pairs = ref;
  q.ref_pixels = refpix;
  LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(q.f1, f1, sizeof(int32_t) * n_pairs, cudaMemcpyHostToDevice, ctx->stream));
  LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(q.f2, f2, sizeof(int32_t) * n_pairs, cudaMemcpyHostToDevice, ctx->stream));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LYA_OK;
}

extern "C" int lya_get_pairs(lya_ctx* ctx, int32_t* f1, int32_t* f2) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_get_pairs: ctx is NULL");
  const int64_t np = ctx->wq.n_pairs;
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  if (np > 0 && f1) LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(f1, ctx->wq.f1, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, ctx->stream));
  if (np > 0 && f2) LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(f2, ctx->wq.f2, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, ctx->stream));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LYA_OK;
}

// ------------------------------------------------------------------ results
__global__ void k_combine(int64_t nslot, int nb, const double* __restrict__ hist, double* __restrict__ out) {
  // hist: [slot][q][2][nb] (hi, lo) -> out [slot][q][nb] = hi + lo
  const int64_t total = nslot * LYA_NQ * (int64_t)nb;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sq = k / nb, b = k - sq * nb;
    out[k] = hist[(sq * 2) * nb + b] + hist[(sq * 2 + 1) * nb + b];
  }
}

extern "C" int lya_corr_get(lya_ctx* ctx, int32_t slot_first, int32_t n, double* hist, uint64_t* counts) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_get: ctx is NULL");
  if (!ctx->have_result) return lya_fail(ctx, LYA_ERR_STATE, "lya_corr_get: no result (call lya_corr_run first)");
  if (slot_first < 0 || n < 0 || slot_first + (int64_t)n > ctx->hist_slots)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_get: slots [%d,%d) outside [0,%d)", slot_first, slot_first + n,
                    ctx->hist_slots);
  if (n == 0) return LYA_OK;
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nb = ctx->hist_nb;
  if (hist) {
    const int64_t need = (int64_t)n * LYA_NQ * nb;
    if (ctx->get_tmp_cap < need) {   // kept for later calls
      lya_free(ctx->get_tmp);
      ctx->get_tmp_cap = 0;
      if (lya_alloc(&ctx->get_tmp, (size_t)need) != cudaSuccess)
        return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_get: device allocation failed");
      ctx->get_tmp_cap = need;
    }
    double* tmp = ctx->get_tmp;
    cudaError_t e = cudaSuccess;
    const double* src = ctx->hist + (size_t)slot_first * LYA_NQ * 2 * nb;
    int blocks = (int)std::min<int64_t>(((int64_t)n * LYA_NQ * nb + 255) / 256, (int64_t)ctx->num_sms * 8);
    k_combine<<<blocks, 256, 0, ctx->stream>>>(n, nb, src, tmp);
    ctx->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hist, tmp, sizeof(double) * (size_t)n * LYA_NQ * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_corr_get: %s", cudaGetErrorString(e));
  }
  if (counts) {
    LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(counts, ctx->counts + (size_t)slot_first * nb,
                                        sizeof(unsigned long long) * (size_t)n * nb, cudaMemcpyDeviceToHost,
                                        ctx->stream));
    LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return LYA_OK;
}

extern "C" int lya_timer(lya_ctx* ctx, int32_t op, double* ms) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_timer: ctx is NULL");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  if (op == 0) {
    LYA_CHECK_CUDA(ctx, cudaEventRecord(ctx->tev0, ctx->stream));
    return LYA_OK;
  }
  if (op != 1 || !ms) return lya_fail(ctx, LYA_ERR_ARG, "lya_timer: op must be 0 or 1 (with ms)");
  LYA_CHECK_CUDA(ctx, cudaEventRecord(ctx->tev1, ctx->stream));
  LYA_CHECK_CUDA(ctx, cudaEventSynchronize(ctx->tev1));
  float f = 0.f;
  LYA_CHECK_CUDA(ctx, cudaEventElapsedTime(&f, ctx->tev0, ctx->tev1));
  *ms = f;
  return LYA_OK;
}

extern "C" int lya_sync(lya_ctx* ctx) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_sync: ctx is NULL");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LYA_OK;
}

extern "C" int lya_stats(lya_ctx* ctx, lya_stats_t* out) {
  if (!ctx || !out) return lya_fail(ctx, LYA_ERR_ARG, "lya_stats: NULL argument");
  lya_resolve_build_timing(ctx);
  *out = ctx->last;
  out->launches = ctx->launches;
  out->n_pairs = ctx->wq.n_pairs;
  out->ref_pairs = ctx->wq.ref_pairs;
  out->ref_pixels = ctx->wq.ref_pixels;
  out->n_slots = ctx->cat.n_slots;
  out->n_forests = (int32_t)ctx->cat.n;
  return LYA_OK;
}
