// Device-side neighbour search: the work queue of forest pairs.
//
// Reference: quasar.neighborhood (forest_class.py:78-98), called by
// two_point_per_pixel for every forest (correlation_procedures_pycuda.py:144):
// healpy.query_disc pre-filters healpix pixels, then a Python loop keeps f2 when
//   (x1*x2 + y1*y2) + z1*z2 > cos(angmax),  name1 != name2,  ra1 < ra2.
// Here one pass over all forests replaces the per-forest Python loops: forests
// are bucketed into declination bands of height >= angmax and sorted by right
// ascension inside each band; one warp per first forest scans the three bands
// that can hold neighbours, restricted to the right-ascension window the
// angular distance allows (with the wrap at ra = 2 pi), and applies the
// reference's exact membership test (FP64, Python's operation order, no FMA).
// The pre-filter is a superset of the disc, so the neighbour set equals the
// reference's; pairs are written grouped by f1 in forest order.
//
// The build allocates nothing once its scratch is sized (the sorts and the scan
// are cub calls on scratch kept in the context) and synchronises once, to size
// the queue from the count pass.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "lya_internal.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int32_t band_of(double dec, double band_h, int64_t nband) {
  int64_t b = (int64_t)floor((dec + M_PI_2) / band_h);
  b = b < 0 ? 0 : (b >= nband ? nband - 1 : b);
  return (int32_t)b;
}

__global__ void k_bands(int64_t n, const double* __restrict__ ra, double* __restrict__ ra_key,
                        int32_t* __restrict__ idx, int* __restrict__ ra_out_of_range) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < n; f += (int64_t)gridDim.x * blockDim.x) {
    ra_key[f] = ra[f];
    idx[f] = (int32_t)f;
    if (!(ra[f] >= 0.0 && ra[f] < 2.0 * M_PI)) atomicExch(ra_out_of_range, 1);
  }
}

// band of every forest, in the ra order of the first sort
__global__ void k_band_keys(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ dec,
                            double band_h, int64_t nband, int32_t* __restrict__ band) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    band[q] = band_of(dec[idx[q]], band_h, nband);
}

// ra in (band, ra) order
__global__ void k_gather_ra(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ ra,
                            double* __restrict__ sra) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    sra[q] = ra[idx[q]];
}

// bstart[b] = first position of band >= b in the sorted band array, b = 0..nband
__global__ void k_band_starts(int64_t n, const int32_t* __restrict__ band, int64_t nband, int64_t* __restrict__ bstart) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= nband; b += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (band[mid] < b) lo = mid + 1; else hi = mid;
    }
    bstart[b] = lo;
  }
}

__device__ __forceinline__ int64_t lower_ra(const double* __restrict__ sra, int64_t lo, int64_t hi, double v) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (sra[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int64_t upper_ra(const double* __restrict__ sra, int64_t lo, int64_t hi, double v) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (sra[mid] <= v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

struct NbrParams {
  int64_t n;
  const double* ra;
  const double* dec;
  const double* ux;
  const double* uy;
  const double* uz;
  const long long* name;
  const int32_t* sidx;     // forests sorted by (band, ra)
  const double* sra;       // their ra
  const int64_t* bstart;   // [nband + 1]
  int64_t nband;
  double band_h, angmax, mumin;
  const int* ra_out_of_range;
  const int32_t* len;         // forest lengths (count pass: reference pixel pairs)
  double* tot;                // count pass: [0] += sum len1*len2, [1] += sum len1+len2
  long long* counts;          // count pass output
  const long long* offsets;   // fill pass input (exclusive scan of counts)
  int32_t* of1;
  int32_t* of2;
};

// One warp per first forest.  FILL = false counts, FILL = true writes.
template <bool FILL>
__global__ void k_neighbours(const NbrParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const bool all_in = *p.ra_out_of_range == 0;
  for (int64_t f1 = gw; f1 < p.n; f1 += nw) {
    const double ra1 = p.ra[f1], dec1 = p.dec[f1];
    const double x1 = p.ux[f1], y1 = p.uy[f1], z1 = p.uz[f1];
    const long long nm1 = p.name[f1];
    const int64_t b1 = band_of(dec1, p.band_h, p.nband);
    // right-ascension half-width of the disc: sin(dra/2) <= sin(angmax/2)/cos(|dec|+angmax)
    const double dlim = fabs(dec1) + p.angmax * (1.0 + 1e-6) + 1e-9;
    bool full = !all_in;
    double dra = 0.0;
    if (dlim >= M_PI_2 - 1e-9) {
      full = true;
    } else {
      const double s = sin(0.5 * p.angmax) / cos(dlim);
      if (s >= 1.0) full = true;
      else {
        dra = 2.0 * asin(s) * (1.0 + 1e-6) + 1e-9;
        if (dra >= M_PI_2) full = true;
      }
    }
    long long cnt = 0;
    double cost = 0.0, pix = 0.0;   // count pass: this lane's accepted pairs
    const double l1 = FILL ? 0.0 : (double)p.len[f1];
    const long long base = FILL ? p.offsets[f1] : 0;
    for (int64_t b = b1 - 1; b <= b1 + 1; ++b) {
      if (b < 0 || b >= p.nband) continue;
      const int64_t lo = p.bstart[b], hi = p.bstart[b + 1];
      int64_t r0s[2], r0e[2];
      int nr = 0;
      if (full) {
        r0s[0] = lo; r0e[0] = hi; nr = 1;
      } else {
        const int64_t p0 = lower_ra(p.sra, lo, hi, ra1);
        const int64_t p1 = upper_ra(p.sra, p0, hi, ra1 + dra);
        r0s[0] = p0; r0e[0] = p1; nr = 1;
        if (ra1 - dra < 0.0) {   // neighbours across ra = 2 pi have larger ra
          r0s[1] = lower_ra(p.sra, lo, hi, ra1 - dra + 2.0 * M_PI);
          r0e[1] = hi;
          if (r0s[1] < p1) r0s[1] = p1;
          nr = 2;
        }
      }
      for (int r = 0; r < nr; ++r) {
        for (int64_t q0 = r0s[r]; q0 < r0e[r]; q0 += 32) {
          const int64_t q = q0 + lane;
          bool acc = false;
          int32_t f2 = 0;
          if (q < r0e[r]) {
            f2 = p.sidx[q];
            const double mu = __dadd_rn(__dadd_rn(__dmul_rn(x1, p.ux[f2]), __dmul_rn(y1, p.uy[f2])),
                                        __dmul_rn(z1, p.uz[f2]));
            acc = mu > p.mumin && nm1 != p.name[f2] && ra1 < p.ra[f2];
          }
          const unsigned bal = __ballot_sync(FULL, acc);
          if (!FILL && acc) {
            const double l2 = (double)p.len[f2];
            cost += l1 * l2;
            pix += l1 + l2;
          }
          if (FILL && acc) {
            const long long pos = base + cnt + __popc(bal & ((1u << lane) - 1u));
            p.of1[pos] = (int32_t)f1;
            p.of2[pos] = f2;
          }
          cnt += __popc(bal);
        }
      }
    }
    if (!FILL) {
      // integer-valued sums below 2^53: exact in any order
      for (int o = 16; o > 0; o >>= 1) {
        cost += __shfl_xor_sync(FULL, cost, o);
        pix += __shfl_xor_sync(FULL, pix, o);
      }
      if (lane == 0) {
        p.counts[f1] = cnt;
        if (cost != 0.0) atomicAdd(p.tot, cost);
        if (pix != 0.0) atomicAdd(p.tot + 1, pix);
      }
    }
  }
}

// keep flag of every work item: its first forest's owner slot is kept
__global__ void k_keep_flags(int64_t n, const int32_t* __restrict__ f1, const int32_t* __restrict__ slot,
                             const uint8_t* __restrict__ keep, long long* __restrict__ flag) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    flag[k] = keep[slot[f1[k]]] ? 1 : 0;
}

// scatter the kept items to their compacted positions (pos = exclusive scan of
// the flags, in the same buffer) and sum their reference pixel pairs
__global__ void k_keep_scatter(int64_t n, const int32_t* __restrict__ f1, const int32_t* __restrict__ f2,
                               const uint8_t* __restrict__ keep, const int32_t* __restrict__ slot,
                               const long long* __restrict__ pos, const int32_t* __restrict__ len,
                               int32_t* __restrict__ o1, int32_t* __restrict__ o2, double* __restrict__ tot) {
  double cost = 0.0, pix = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = f1[k];
    if (keep[slot[a]]) {
      const int32_t b = f2[k];
      o1[pos[k]] = a;
      o2[pos[k]] = b;
      const double l1 = (double)len[a], l2 = (double)len[b];
      cost += l1 * l2;
      pix += l1 + l2;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    cost += __shfl_xor_sync(FULL, cost, o);
    pix += __shfl_xor_sync(FULL, pix, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (cost != 0.0) atomicAdd(tot, cost);
    if (pix != 0.0) atomicAdd(tot + 1, pix);
  }
}

}  // namespace

// Scratch for a build over n forests and nband declination bands, kept
// between builds when large enough.
static cudaError_t nbr_reserve(lya_ctx* ctx, int64_t n, int64_t nband) {
  NbrScratch& S = ctx->nbr;
  cudaError_t e = cudaSuccess;
  if (!S.h_out) {
    e = cudaMallocHost((void**)&S.h_out, sizeof(long long) * 4);
    if (e == cudaSuccess) e = cudaEventCreate(&S.ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&S.ev1);
    if (e == cudaSuccess) e = lya_alloc(&S.flag, 1);
    if (e == cudaSuccess) e = lya_alloc(&S.tot, 2);
    if (e != cudaSuccess) return e;
  }
  if (S.band && n <= S.cap_n && nband <= S.cap_band) return cudaSuccess;
  lya_free(S.band); lya_free(S.band2); lya_free(S.sidx); lya_free(S.sidx2); lya_free(S.sra); lya_free(S.sra2);
  lya_free(S.bstart); lya_free(S.counts); lya_free(S.offsets);
  if (S.tmp) cudaFree(S.tmp);
  S.tmp = nullptr;
  S.tmp_bytes = 0;
  S.cap_n = 0;
  S.cap_band = 0;
  e = lya_alloc(&S.band, n);
  if (e == cudaSuccess) e = lya_alloc(&S.band2, n);
  if (e == cudaSuccess) e = lya_alloc(&S.sidx, n);
  if (e == cudaSuccess) e = lya_alloc(&S.sidx2, n);
  if (e == cudaSuccess) e = lya_alloc(&S.sra, n);
  if (e == cudaSuccess) e = lya_alloc(&S.sra2, n);
  if (e == cudaSuccess) e = lya_alloc(&S.bstart, nband + 1);
  if (e == cudaSuccess) e = lya_alloc(&S.counts, n + 1);
  if (e == cudaSuccess) e = lya_alloc(&S.offsets, n + 1);
  // cub scratch: the larger of the two sorts and the scan
  size_t b1 = 0, b2 = 0, b3 = 0;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(nullptr, b1, S.sra2, S.sra, S.sidx2, S.sidx, (int)n, 0, 64, ctx->stream);
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(nullptr, b2, S.band2, S.band, S.sidx2, S.sidx, (int)n, 0, 32, ctx->stream);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, b3, S.counts, S.offsets, (int)(n + 1), ctx->stream);
  const size_t bytes = std::max(b1, std::max(b2, b3));
  if (e == cudaSuccess) e = cudaMalloc(&S.tmp, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return e;
  S.tmp_bytes = std::max<size_t>(bytes, 16);
  S.cap_n = n;
  S.cap_band = nband;
  return cudaSuccess;
}

void lya_resolve_build_timing(lya_ctx* ctx) {
  NbrScratch& S = ctx->nbr;
  if (!S.timing_pending) return;
  float ms = 0.f;
  if (cudaEventSynchronize(S.ev1) == cudaSuccess && cudaEventElapsedTime(&ms, S.ev0, S.ev1) == cudaSuccess)
    ctx->last.build_ms = ms;
  S.timing_pending = false;
}

int lya_build_queue(lya_ctx* ctx, double angmax, double mumin) {
  const int64_t n = ctx->cat.n;
  cudaStream_t s = ctx->stream;
  const double h = angmax * (1.0 + 1e-6) + 1e-9;
  const int64_t nband = (int64_t)std::ceil(M_PI / h) + 2;
  if (n >= (int64_t)INT32_MAX - 1) return lya_fail(ctx, LYA_ERR_ARG, "lya_build_pairs: too many forests");
  lya_resolve_build_timing(ctx);
  cudaError_t e = nbr_reserve(ctx, n, nband);
  if (e != cudaSuccess) {
    lya_free_nbr_scratch(ctx->nbr);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_build_pairs: allocation of the search scratch failed (%s)",
                    cudaGetErrorString(e));
  }
  NbrScratch& S = ctx->nbr;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  const int nb_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nband + 1 + 127) / 128, 64));
  NbrParams p;
  p.n = n; p.ra = ctx->cat.ra; p.dec = ctx->cat.dec; p.ux = ctx->cat.ux; p.uy = ctx->cat.uy; p.uz = ctx->cat.uz;
  p.name = ctx->cat.name; p.sidx = S.sidx; p.sra = S.sra; p.bstart = S.bstart; p.nband = nband; p.band_h = h;
  p.angmax = angmax; p.mumin = mumin; p.ra_out_of_range = S.flag; p.len = ctx->cat.len; p.tot = S.tot;
  p.counts = S.counts; p.offsets = S.offsets; p.of1 = nullptr; p.of2 = nullptr;
  const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256, (int64_t)ctx->num_sms * 32));
  size_t tb = S.tmp_bytes;
  e = cudaEventRecord(S.ev0, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(S.flag, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(S.tot, 0, 2 * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(S.counts, 0, sizeof(long long) * (n + 1), s);
  if (e == cudaSuccess) {
    k_bands<<<blocks, 256, 0, s>>>(n, ctx->cat.ra, S.sra2, S.sidx2, S.flag);
    e = cudaGetLastError();
  }
  // order by (band, ra): stable radix sort by ra, then stable radix sort by band
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(S.tmp, tb, S.sra2, S.sra, S.sidx2, S.sidx, (int)n, 0, 64, s);
  if (e == cudaSuccess) {
    k_band_keys<<<blocks, 256, 0, s>>>(n, S.sidx, ctx->cat.dec, h, nband, S.band2);
    e = cudaGetLastError();
  }
  tb = S.tmp_bytes;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(S.tmp, tb, S.band2, S.band, S.sidx, S.sidx2, (int)n, 0, 32, s);
  if (e == cudaSuccess) {
    std::swap(S.sidx, S.sidx2);   // sidx: forests in (band, ra) order
    p.sidx = S.sidx;
    k_gather_ra<<<blocks, 256, 0, s>>>(n, S.sidx, ctx->cat.ra, S.sra);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_band_starts<<<nb_blocks, 128, 0, s>>>(n, S.band, nband, S.bstart);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_neighbours<false><<<nblk, 256, 0, s>>>(p);
    e = cudaGetLastError();
  }
  tb = S.tmp_bytes;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(S.tmp, tb, S.counts, S.offsets, (int)(n + 1), s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(S.h_out, S.offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(S.h_out + 1, S.tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // the one synchronisation: the queue's size
  // k_bands, k_band_keys, k_gather_ra, k_band_starts, the count pass (the cub sorts and scan are library kernels)
  ctx->launches += 5;
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_build_pairs: %s", cudaGetErrorString(e));
  const long long npairs = S.h_out[0];
  double ref[2];
  memcpy(ref, S.h_out + 1, sizeof(ref));
  ctx->wq.n_pairs = 0;
  e = lya_queue_reserve(ctx->wq, npairs);
  if (e != cudaSuccess) {
    lya_free_queue(ctx->wq);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_build_pairs: queue allocation failed (%lld pairs)", npairs);
  }
  p.of1 = ctx->wq.f1; p.of2 = ctx->wq.f2;
  k_neighbours<true><<<nblk, 256, 0, s>>>(p);
  ctx->launches++;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(S.ev1, s);
  if (e != cudaSuccess) {
    lya_free_queue(ctx->wq);
    return lya_fail(ctx, LYA_ERR_CUDA, "lya_build_pairs: %s", cudaGetErrorString(e));
  }
  S.timing_pending = true;   // build_ms is read once the fill pass has run (lya_stats)
  ctx->wq.n_pairs = npairs;
  ctx->wq.ref_pairs = ref[0];
  ctx->wq.ref_pixels = ref[1];
  return LYA_OK;
}

extern "C" int lya_build_pairs(lya_ctx* ctx, double angmax, double mumin, int64_t* n_pairs_out) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_build_pairs: ctx is NULL");
  if (!(angmax > 0.0) || !(angmax < M_PI)) return lya_fail(ctx, LYA_ERR_ARG, "lya_build_pairs: angmax %g outside (0, pi)", angmax);
  if (ctx->cat.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_build_pairs: no forests uploaded");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->have_result = false;
  const int rc = lya_build_queue(ctx, angmax, mumin);
  if (rc == LYA_OK && n_pairs_out) *n_pairs_out = ctx->wq.n_pairs;
  return rc;
}

extern "C" int lya_select_slots(lya_ctx* ctx, const uint8_t* keep) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_select_slots: ctx is NULL");
  if (!keep) return lya_fail(ctx, LYA_ERR_ARG, "lya_select_slots: keep is NULL");
  if (ctx->cat.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_select_slots: no forests uploaded");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  lya_resolve_build_timing(ctx);
  ctx->have_result = false;
  WorkQueue& q = ctx->wq;
  const int64_t n = q.n_pairs;
  const int32_t nslots = ctx->cat.n_slots;
  SelectScratch& S = ctx->sel;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaSuccess;
  // scratch: keep flags per slot, per-item flags/positions, the compacted copy
  if (!S.h_out) e = cudaMallocHost((void**)&S.h_out, sizeof(double) * 3);
  if (e == cudaSuccess && !S.tot) e = lya_alloc(&S.tot, 2);
  if (e == cudaSuccess && S.keep_cap < nslots) {
    lya_free(S.keep);
    S.keep_cap = 0;
    e = lya_alloc(&S.keep, (size_t)std::max<int32_t>(nslots, 1));
    if (e == cudaSuccess) S.keep_cap = nslots;
  }
  if (e == cudaSuccess && S.cap < std::max<int64_t>(n, 1)) {
    lya_free(S.pos); lya_free(S.o1); lya_free(S.o2);
    if (S.tmp) cudaFree(S.tmp);
    S.tmp = nullptr; S.tmp_bytes = 0; S.cap = 0;
    const int64_t c = std::max<int64_t>(n, 1);
    e = lya_alloc(&S.pos, (size_t)c + 1);
    if (e == cudaSuccess) e = lya_alloc(&S.o1, (size_t)c);
    if (e == cudaSuccess) e = lya_alloc(&S.o2, (size_t)c);
    size_t b = 0;
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, b, S.pos, S.pos, (int)(c + 1), s);
    if (e == cudaSuccess) e = cudaMalloc(&S.tmp, std::max<size_t>(b, 16));
    if (e == cudaSuccess) { S.tmp_bytes = std::max<size_t>(b, 16); S.cap = c; }
  }
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_ALLOC, "lya_select_slots: allocation failed (%s)",
                                        cudaGetErrorString(e));
  if (n >= (int64_t)INT32_MAX) return lya_fail(ctx, LYA_ERR_ARG, "lya_select_slots: queue too long");
  e = cudaMemcpyAsync(S.keep, keep, (size_t)nslots, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(S.tot, 0, 2 * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(S.pos + n, 0, sizeof(long long), s);
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  if (e == cudaSuccess && n > 0) {
    k_keep_flags<<<blocks, 256, 0, s>>>(n, q.f1, ctx->cat.slot, S.keep, S.pos);
    e = cudaGetLastError();
    size_t tb = S.tmp_bytes;
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(S.tmp, tb, S.pos, S.pos, (int)(n + 1), s);
    if (e == cudaSuccess) {
      k_keep_scatter<<<blocks, 256, 0, s>>>(n, q.f1, q.f2, S.keep, ctx->cat.slot, S.pos, ctx->cat.len, S.o1, S.o2,
                                            S.tot);
      e = cudaGetLastError();
    }
    ctx->launches += 2;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(S.h_out, S.pos + n, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(S.h_out + 1, S.tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  long long kept = 0;
  if (e == cudaSuccess) memcpy(&kept, S.h_out, sizeof(kept));
  if (e == cudaSuccess && kept > 0) e = cudaMemcpyAsync(q.f1, S.o1, sizeof(int32_t) * kept, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && kept > 0) e = cudaMemcpyAsync(q.f2, S.o2, sizeof(int32_t) * kept, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_select_slots: %s", cudaGetErrorString(e));
  q.n_pairs = kept;
  q.ref_pairs = S.h_out[1];
  q.ref_pixels = S.h_out[2];
  return LYA_OK;
}
