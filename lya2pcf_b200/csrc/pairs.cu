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
#include <thrust/binary_search.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/tuple.h>

#include <algorithm>
#include <cmath>

#include "lya_internal.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__global__ void k_bands(int64_t n, const double* __restrict__ ra, const double* __restrict__ dec, double band_h,
                        int64_t nband, int32_t* __restrict__ band, double* __restrict__ ra_key,
                        int32_t* __restrict__ idx, int* __restrict__ ra_out_of_range) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < n; f += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = (int64_t)floor((dec[f] + M_PI_2) / band_h);
    b = b < 0 ? 0 : (b >= nband ? nband - 1 : b);
    band[f] = (int32_t)b;
    ra_key[f] = ra[f];
    idx[f] = (int32_t)f;
    if (!(ra[f] >= 0.0 && ra[f] < 2.0 * M_PI)) atomicExch(ra_out_of_range, 1);
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
    int64_t b1 = (int64_t)floor((dec1 + M_PI_2) / p.band_h);
    b1 = b1 < 0 ? 0 : (b1 >= p.nband ? p.nband - 1 : b1);
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
          if (FILL && acc) {
            const long long pos = base + cnt + __popc(bal & ((1u << lane) - 1u));
            p.of1[pos] = (int32_t)f1;
            p.of2[pos] = f2;
          }
          cnt += __popc(bal);
        }
      }
    }
    if (!FILL && lane == 0) p.counts[f1] = cnt;
  }
}

// out[0] += sum len1*len2 (reference pixel pairs), out[1] += sum len1+len2
__global__ void k_pair_cost(int64_t n, const int32_t* __restrict__ f1, const int32_t* __restrict__ f2,
                            const int32_t* __restrict__ len, double* __restrict__ out) {
  double acc = 0.0, pix = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double l1 = (double)len[f1[k]], l2 = (double)len[f2[k]];
    acc += l1 * l2;
    pix += l1 + l2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_xor_sync(FULL, acc, o);
    pix += __shfl_xor_sync(FULL, pix, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, acc);
    atomicAdd(out + 1, pix);
  }
}

}  // namespace

int lya_build_queue(lya_ctx* ctx, double angmax, double mumin) {
  const int64_t n = ctx->cat.n;
  cudaStream_t s = ctx->stream;
  auto pol = thrust::cuda::par.on(s);
  const double h = angmax * (1.0 + 1e-6) + 1e-9;
  const int64_t nband = (int64_t)std::ceil(M_PI / h) + 2;

  int32_t *band = nullptr, *sidx = nullptr;
  double *sra = nullptr, *tot = nullptr;
  int64_t* bstart = nullptr;
  long long *counts = nullptr, *offsets = nullptr;
  int* flag = nullptr;
  cudaError_t e = lya_alloc(&band, n);
  if (e == cudaSuccess) e = lya_alloc(&sidx, n);
  if (e == cudaSuccess) e = lya_alloc(&sra, n);
  if (e == cudaSuccess) e = lya_alloc(&bstart, nband + 1);
  if (e == cudaSuccess) e = lya_alloc(&counts, n + 1);
  if (e == cudaSuccess) e = lya_alloc(&offsets, n + 1);
  if (e == cudaSuccess) e = lya_alloc(&flag, 1);
  if (e == cudaSuccess) e = lya_alloc(&tot, 2);
  auto cleanup = [&]() {
    lya_free(band); lya_free(sidx); lya_free(sra); lya_free(bstart); lya_free(counts); lya_free(offsets);
    lya_free(flag); lya_free(tot);
  };
  if (e != cudaSuccess) {
    cleanup();
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_build_pairs: allocation failed");
  }
  LYA_CHECK_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
  cudaMemsetAsync(flag, 0, sizeof(int), s);
  cudaMemsetAsync(tot, 0, 2 * sizeof(double), s);
  cudaMemsetAsync(counts, 0, sizeof(long long) * (n + 1), s);
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  k_bands<<<blocks, 256, 0, s>>>(n, ctx->cat.ra, ctx->cat.dec, h, nband, band, sra, sidx, flag);
  ctx->launches++;
  // order by (band, ra): stable sort by ra, then stable sort by band
  thrust::stable_sort_by_key(pol, sra, sra + n, thrust::make_zip_iterator(thrust::make_tuple(sidx, band)));
  thrust::stable_sort_by_key(pol, band, band + n, thrust::make_zip_iterator(thrust::make_tuple(sidx, sra)));
  thrust::lower_bound(pol, band, band + n, thrust::counting_iterator<int32_t>(0),
                      thrust::counting_iterator<int32_t>((int32_t)nband + 1), bstart);

  NbrParams p;
  p.n = n; p.ra = ctx->cat.ra; p.dec = ctx->cat.dec; p.ux = ctx->cat.ux; p.uy = ctx->cat.uy; p.uz = ctx->cat.uz;
  p.name = ctx->cat.name; p.sidx = sidx; p.sra = sra; p.bstart = bstart; p.nband = nband; p.band_h = h;
  p.angmax = angmax; p.mumin = mumin; p.ra_out_of_range = flag; p.counts = counts; p.offsets = offsets;
  p.of1 = nullptr; p.of2 = nullptr;
  const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256, (int64_t)ctx->num_sms * 32));
  k_neighbours<false><<<nblk, 256, 0, s>>>(p);
  ctx->launches++;
  thrust::exclusive_scan(pol, counts, counts + n + 1, offsets);
  long long npairs = 0;
  e = cudaMemcpyAsync(&npairs, offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cleanup();
    return lya_fail(ctx, LYA_ERR_CUDA, "lya_build_pairs: %s", cudaGetErrorString(e));
  }
  ctx->wq.n_pairs = 0;
  e = lya_queue_reserve(ctx->wq, npairs);
  if (e != cudaSuccess) {
    cleanup();
    lya_free_queue(ctx->wq);
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_build_pairs: queue allocation failed (%lld pairs)", npairs);
  }
  p.of1 = ctx->wq.f1; p.of2 = ctx->wq.f2;
  k_neighbours<true><<<nblk, 256, 0, s>>>(p);
  ctx->launches++;
  if (npairs > 0) {
    const int cb = (int)std::min<int64_t>((npairs + 255) / 256, (int64_t)ctx->num_sms * 8);
    k_pair_cost<<<cb, 256, 0, s>>>(npairs, ctx->wq.f1, ctx->wq.f2, ctx->cat.len, tot);
    ctx->launches++;
  }
  double ref[2] = {0.0, 0.0};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ref, tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  cleanup();
  if (e != cudaSuccess) {
    lya_free_queue(ctx->wq);
    return lya_fail(ctx, LYA_ERR_CUDA, "lya_build_pairs: %s", cudaGetErrorString(e));
  }
  ctx->wq.n_pairs = npairs;
  ctx->wq.ref_pairs = ref[0];
  ctx->wq.ref_pixels = ref[1];
  ctx->last.build_ms = ms;
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
