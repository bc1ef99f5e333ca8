// Covariance post-processing of the per-pixel correlation estimates.
//
// Reference: cov and cov_smooth (post_processing.py:30-91), numba loops that
// form, for every pair of bins (a, b),
//   C_ab = sum_p w_pa (xi_pa - m_a) w_pb (xi_pb - m_b) / (W_a W_b),
//   m_a = sum_p xi_pa w_pa / W_a,   W_a = sum_p w_pa,
// over the owner pixels p (xi = DW/W of a pixel, 0 where W = 0,
// post_processing.py:139-147), and then average the correlation matrix
// C_ab / sqrt(C_aa C_bb) over pairs of bins with the same (|r_par step|,
// |r_perp step|) (bin labels from bin_coordinates, post_processing.py:13-28).
//
// B200 form: the centred, weighted estimates Y_pa = w_pa (xi_pa - m_a) are
// formed once and C = Y^T Y / (W W^T) is a dense FP64 Gram matrix computed on
// the tensor cores (mma.sync m8n8k4 f64; FP64 has no tcgen05 kind): 64 x 64
// output tiles of the upper triangle, rows of Y staged in shared memory 32 at a
// time, warp w owning tile row w of a tile.  The step averages are per-CTA
// shared-memory sums flushed with FP64 atomics.  A bin whose weights sum to 0
// is reported (the reference's numba code raises ZeroDivisionError there).
#include <algorithm>
#include <cmath>
#include <vector>

#include "lya_internal.cuh"

namespace {

constexpr int CT = 64;         // output tile (bins x bins)
constexpr int KC = 32;         // rows of Y staged per chunk (a multiple of 4)
constexpr int SPAD = CT + 4;   // staged row stride (doubles): conflict-free fragment loads
constexpr int GT = 256;        // threads of the Gram kernel (8 warps = 8 tile rows)

// W_b and m_b, one thread per bin, rows in order.
__global__ void k_cov_stats(int64_t n, int nb, const double* __restrict__ xi, const double* __restrict__ w,
                            double* __restrict__ W, double* __restrict__ mean, unsigned long long* __restrict__ zero) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double sw = 0.0, sxw = 0.0;
    for (int64_t p = 0; p < n; ++p) {
      const double wv = w[p * nb + b];
      sw += wv;
      sxw += xi[p * nb + b] * wv;
    }
    W[b] = sw;
    mean[b] = sw != 0.0 ? sxw / sw : 0.0;
    if (sw == 0.0) atomicAdd(zero, 1ull);
  }
}

// xi = DW / W (0 where W = 0) and w = W of every owner slot, from the
// compensated per-slot histograms of the last correlation run.
__global__ void k_cov_from_hist(int64_t nslot, int nb, const double* __restrict__ hist, double* __restrict__ xi,
                                double* __restrict__ w) {
  const int64_t total = nslot * (int64_t)nb;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = k / nb, b = k - s * nb;
    const double* h = hist + s * LYA_NQ * 2 * nb;   // [q][hi, lo][nb]
    const double W = h[b] + h[nb + b];
    const double DW = h[2 * nb + b] + h[3 * nb + b];
    w[k] = W;
    xi[k] = W != 0.0 ? DW / W : 0.0;
  }
}

__global__ void k_cov_center(int64_t n, int nb, const double* __restrict__ xi, const double* __restrict__ w,
                             const double* __restrict__ mean, double* __restrict__ y) {
  const int64_t total = n * (int64_t)nb;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(k % nb);
    y[k] = w[k] * (xi[k] - mean[b]);
  }
}

// C = Y^T Y / (W W^T), tile (ta, tb) with ta <= tb, mirrored.
__global__ void __launch_bounds__(GT) k_cov_gram(int64_t n, int nb, const double* __restrict__ y,
                                                 const double* __restrict__ W, double* __restrict__ cov) {
  __shared__ __align__(16) double Ya[KC * SPAD];
  __shared__ __align__(16) double Yb[KC * SPAD];
  const int ntile = (nb + CT - 1) / CT;
  const int ta = blockIdx.y, tb = blockIdx.x;
  if (ta > tb || ta >= ntile || tb >= ntile) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = lane >> 2, kq = lane & 3;
  const int a0 = ta * CT, b0 = tb * CT;
  double acc[8][2];
#pragma unroll
  for (int c = 0; c < 8; ++c) { acc[c][0] = 0.0; acc[c][1] = 0.0; }
  for (int64_t p0 = 0; p0 < n; p0 += KC) {
    for (int e = tid; e < KC * CT; e += GT) {
      const int r = e / CT, c = e - r * CT;
      const int64_t p = p0 + r;
      const bool rowok = p < n;
      Ya[r * SPAD + c] = (rowok && a0 + c < nb) ? y[p * nb + a0 + c] : 0.0;
      Yb[r * SPAD + c] = (rowok && b0 + c < nb) ? y[p * nb + b0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int r0 = 0; r0 < KC; r0 += 4) {
      const int ra = (r0 + kq) * SPAD;
      const double av = Ya[ra + 8 * warp + grp];
#pragma unroll
      for (int c = 0; c < 8; ++c) lya_dmma_8x8x4(acc[c][0], acc[c][1], av, Yb[ra + 8 * c + grp]);
    }
    __syncthreads();
  }
  const int a = a0 + 8 * warp + grp;
  if (a >= nb) return;
  const double Wa = W[a];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int b = b0 + 8 * c + 2 * kq + i;
      if (b >= nb) continue;
      const double v = acc[c][i] / (Wa * W[b]);
      cov[(size_t)a * nb + b] = v;
      if (ta != tb) cov[(size_t)b * nb + a] = v;
    }
  }
}

// Sums and counts of the correlation over the steps (|bp_a - bp_b|,
// |bt_a - bt_b|) of the pairs a < b; a block per range of rows a.
__global__ void k_cov_steps(int nb, int np, int nt, const double* __restrict__ cov, double* __restrict__ ssum,
                            double* __restrict__ scnt) {
  extern __shared__ __align__(16) double sm[];
  double* s_sum = sm;             // [np * nt]
  double* s_cnt = sm + np * nt;   // [np * nt]
  for (int k = threadIdx.x; k < 2 * np * nt; k += blockDim.x) sm[k] = 0.0;
  __syncthreads();
  for (int a = blockIdx.x; a < nb; a += gridDim.x) {
    const int pa = a / nt, qa = a - pa * nt;
    const double va = cov[(size_t)a * nb + a];
    for (int b = a + 1 + threadIdx.x; b < nb; b += blockDim.x) {
      const int pb = b / nt, qb = b - pb * nt;
      const double vb = cov[(size_t)b * nb + b];
      const double corr = cov[(size_t)a * nb + b] / sqrt(va * vb);
      const int st = abs(pb - pa) * nt + abs(qb - qa);
      atomicAdd(&s_sum[st], corr);
      atomicAdd(&s_cnt[st], 1.0);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < np * nt; k += blockDim.x) {
    if (s_cnt[k] != 0.0) {
      atomicAdd(&ssum[k], s_sum[k]);
      atomicAdd(&scnt[k], s_cnt[k]);
    }
  }
}

__global__ void k_cov_smooth(int nb, int nt, const double* __restrict__ cov, const double* __restrict__ ssum,
                             const double* __restrict__ scnt, double* __restrict__ out) {
  const int64_t total = (int64_t)nb * nb;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(k / nb), b = (int)(k - (int64_t)a * nb);
    if (a == b) { out[k] = cov[k]; continue; }
    const int pa = a / nt, qa = a - pa * nt, pb = b / nt, qb = b - pb * nt;
    const int st = abs(pb - pa) * nt + abs(qb - qa);
    const double norm = sqrt(cov[(size_t)a * nb + a] * cov[(size_t)b * nb + b]);
    out[k] = ssum[st] / scnt[st] * norm;
  }
}

__global__ void k_count_zero_diag(int nb, const double* __restrict__ cov, unsigned long long* __restrict__ zero) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
    if (cov[(size_t)b * nb + b] == 0.0) atomicAdd(zero, 1ull);
}

}  // namespace

extern "C" int lya_covariance(lya_ctx* ctx, int64_t n_rows, const double* xi, const double* w, double* mean,
                              double* cov) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_covariance: ctx is NULL");
  if (!ctx->bins_set) return lya_fail(ctx, LYA_ERR_STATE, "lya_covariance: call lya_set_bins first");
  const bool from_run = xi == nullptr && w == nullptr;
  if (!from_run && (!xi || !w)) return lya_fail(ctx, LYA_ERR_ARG, "lya_covariance: give both xi and w, or neither");
  if (from_run && !ctx->have_result)
    return lya_fail(ctx, LYA_ERR_STATE, "lya_covariance: no correlation run to take the histograms from");
  const int nb = ctx->np * ctx->nt;
  const int64_t n = from_run ? (int64_t)ctx->cat.n_slots : n_rows;
  if (n <= 0) return lya_fail(ctx, LYA_ERR_ARG, "lya_covariance: need at least one row (got %lld)", (long long)n);
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  if (ctx->cov_nb != nb || !ctx->cov) {
    lya_free(ctx->cov);
    ctx->cov_nb = 0;
    if (lya_alloc(&ctx->cov, (size_t)nb * nb) != cudaSuccess)
      return lya_fail(ctx, LYA_ERR_ALLOC, "lya_covariance: device allocation failed");
    ctx->cov_nb = nb;
  }
  ctx->have_cov = false;
  double *d_xi = nullptr, *d_w = nullptr, *d_y = nullptr, *d_W = nullptr, *d_mean = nullptr;
  unsigned long long* d_zero = nullptr;
  cudaError_t e = lya_alloc(&d_xi, (size_t)n * nb);
  if (e == cudaSuccess) e = lya_alloc(&d_w, (size_t)n * nb);
  if (e == cudaSuccess) e = lya_alloc(&d_y, (size_t)n * nb);
  if (e == cudaSuccess) e = lya_alloc(&d_W, nb);
  if (e == cudaSuccess) e = lya_alloc(&d_mean, nb);
  if (e == cudaSuccess) e = lya_alloc(&d_zero, 1);
  auto cleanup = [&]() { lya_free(d_xi); lya_free(d_w); lya_free(d_y); lya_free(d_W); lya_free(d_mean); lya_free(d_zero); };
  if (e != cudaSuccess) {
    cleanup();
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_covariance: device allocation failed");
  }
  const int blocks = ctx->num_sms * 8;
  if (from_run) {
    k_cov_from_hist<<<blocks, 256, 0, s>>>(n, nb, ctx->hist, d_xi, d_w);
    ctx->launches++;
  } else {
    e = cudaMemcpyAsync(d_xi, xi, sizeof(double) * (size_t)n * nb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_w, w, sizeof(double) * (size_t)n * nb, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(d_zero, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
  if (e == cudaSuccess) {
    k_cov_stats<<<(nb + 127) / 128, 128, 0, s>>>(n, nb, d_xi, d_w, d_W, d_mean, d_zero);
    k_cov_center<<<blocks, 256, 0, s>>>(n, nb, d_xi, d_w, d_mean, d_y);
    const int nt_ = (nb + CT - 1) / CT;
    k_cov_gram<<<dim3(nt_, nt_), GT, 0, s>>>(n, nb, d_y, d_W, ctx->cov);
    ctx->launches += 3;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
  unsigned long long nzero = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nzero, d_zero, sizeof(nzero), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && mean) e = cudaMemcpyAsync(mean, d_mean, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && cov)
    e = cudaMemcpyAsync(cov, ctx->cov, sizeof(double) * (size_t)nb * nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  cleanup();
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_covariance: %s", cudaGetErrorString(e));
  ctx->last.kernel_ms = ms;
  if (nzero) return lya_fail(ctx, LYA_ERR_DATA, "lya_covariance: %llu bins have zero total weight", nzero);
  ctx->have_cov = true;
  return LYA_OK;
}

extern "C" int lya_covariance_smooth(lya_ctx* ctx, const double* cov, double* cov_smooth, int32_t* smoothed) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_covariance_smooth: ctx is NULL");
  if (!ctx->bins_set) return lya_fail(ctx, LYA_ERR_STATE, "lya_covariance_smooth: call lya_set_bins first");
  if (!cov_smooth) return lya_fail(ctx, LYA_ERR_ARG, "lya_covariance_smooth: cov_smooth is NULL");
  const int np = ctx->np, nt = ctx->nt, nb = np * nt;
  if (!cov && (!ctx->have_cov || ctx->cov_nb != nb))
    return lya_fail(ctx, LYA_ERR_STATE, "lya_covariance_smooth: no covariance from lya_covariance");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  double *d_cov = nullptr, *d_out = nullptr, *d_sum = nullptr;
  unsigned long long* d_zero = nullptr;
  cudaError_t e = cudaSuccess;
  if (cov) e = lya_alloc(&d_cov, (size_t)nb * nb);
  if (e == cudaSuccess) e = lya_alloc(&d_out, (size_t)nb * nb);
  if (e == cudaSuccess) e = lya_alloc(&d_sum, 2 * (size_t)nb);
  if (e == cudaSuccess) e = lya_alloc(&d_zero, 1);
  auto cleanup = [&]() { lya_free(d_cov); lya_free(d_out); lya_free(d_sum); lya_free(d_zero); };
  if (e != cudaSuccess) {
    cleanup();
    return lya_fail(ctx, LYA_ERR_ALLOC, "lya_covariance_smooth: device allocation failed");
  }
  const double* src = cov ? d_cov : ctx->cov;
  if (cov) e = cudaMemcpyAsync(d_cov, cov, sizeof(double) * (size_t)nb * nb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_zero, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_sum, 0, sizeof(double) * 2 * nb, s);
  if (e == cudaSuccess) {
    k_count_zero_diag<<<(nb + 255) / 256, 256, 0, s>>>(nb, src, d_zero);
    ctx->launches++;
    e = cudaGetLastError();
  }
  unsigned long long nzero = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nzero, d_zero, sizeof(nzero), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && nzero == 0) {
    // a zero variance leaves the covariance unsmoothed, as the reference does
    const size_t smem = sizeof(double) * 2 * (size_t)nb;
    if (smem > 227 * 1024) {
      cleanup();
      return lya_fail(ctx, LYA_ERR_ARG, "lya_covariance_smooth: %d bins exceed the step table", nb);
    }
    e = cudaFuncSetAttribute(k_cov_steps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      k_cov_steps<<<std::min(nb, ctx->num_sms * 2), 256, smem, s>>>(nb, np, nt, src, d_sum, d_sum + nb);
      k_cov_smooth<<<ctx->num_sms * 8, 256, 0, s>>>(nb, nt, src, d_sum, d_sum + nb, d_out);
      ctx->launches += 2;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cov_smooth, d_out, sizeof(double) * (size_t)nb * nb, cudaMemcpyDeviceToHost, s);
  } else if (e == cudaSuccess) {
    e = cudaMemcpyAsync(cov_smooth, src, sizeof(double) * (size_t)nb * nb, cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_covariance_smooth: %s", cudaGetErrorString(e));
  if (smoothed) *smoothed = nzero == 0 ? 1 : 0;
  return LYA_OK;
}
