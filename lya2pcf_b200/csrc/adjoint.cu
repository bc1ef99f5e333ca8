// Adjoint of the pair histograms (no reference counterpart).
//
// Loss L = sum_b g_b xi_b with xi_b = DW_b / W_b (totals over all owner slots
// of the last lya_corr_run), pair bins held fixed.  For every in-range pixel
// pair (i, j) in bin b:
//   dL/d(dw_i) += (g_b / W_b) dw_j            dL/d(w_i) += -(g_b xi_b / W_b) w_j
// and symmetrically for j.  Bins with W_b == 0 contribute nothing (xi_b = 0,
// as post_processing.py:147 defines it).
//
// Gather form: the work queue is walked in both directions, (f1, f2) and
// (f2, f1); a warp owns the first forest of each item and sums the gradient of
// its pixels in registers (one lane per pixel i, walking j), so no pixel pair
// scatters into memory.  The pair bin is symmetric under the swap (|dc1-dc2|,
// dc1+dc2 and the FMA-ordered cos12 are), so both directions see the same bin.
// Bins are evaluated with the reference FP64 formula.  With sorted dc, the j
// loop is limited to the window where rp < rpmax and rt < rtmax.
#include <algorithm>
#include <cmath>

#include "lya_internal.cuh"

namespace {

struct AdjParams {
  const double* __restrict__ dc;
  const double* __restrict__ w;
  const double* __restrict__ dw;
  const int64_t* __restrict__ pstart;
  const int32_t* __restrict__ len;
  const uint8_t* __restrict__ sorted;
  const double* __restrict__ ux;
  const double* __restrict__ uy;
  const double* __restrict__ uz;
  const int32_t* __restrict__ f1;
  const int32_t* __restrict__ f2;
  int64_t n_items;
  double binner_rp, binner_rt;
  int np, nt, nb, cos_variant;
  const double* __restrict__ coef;   // [2][nb]: g/W, -g xi/W
  double* __restrict__ g_dw;         // padded pixel layout
  double* __restrict__ g_w;
};

__global__ void k_coef(int nslots, int nb, const double* __restrict__ hist, const double* __restrict__ g,
                       double* __restrict__ coef) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double W = 0.0, DW = 0.0;
    for (int s = 0; s < nslots; ++s) {
      const double* h = hist + (size_t)s * LYA_NQ * 2 * nb;
      W += h[(0 * 2 + 0) * nb + b] + h[(0 * 2 + 1) * nb + b];
      DW += h[(1 * 2 + 0) * nb + b] + h[(1 * 2 + 1) * nb + b];
    }
    double cdw = 0.0, cw = 0.0;
    if (W != 0.0) {
      cdw = g[b] / W;
      cw = -g[b] * (DW / W) / W;
    }
    coef[b] = cdw;
    coef[nb + b] = cw;
  }
}

// Totals over all slots of the last run: W[b] and DW[b] (hi + lo of each slot).
__global__ void k_totals(int nslots, int nb, const double* __restrict__ hist, double* __restrict__ W,
                         double* __restrict__ DW) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double w = 0.0, dw = 0.0;
    for (int s = 0; s < nslots; ++s) {
      const double* h = hist + (size_t)s * LYA_NQ * 2 * nb;
      w += h[(0 * 2 + 0) * nb + b] + h[(0 * 2 + 1) * nb + b];
      dw += h[(1 * 2 + 0) * nb + b] + h[(1 * 2 + 1) * nb + b];
    }
    W[b] = w;
    DW[b] = dw;
  }
}

// Reversed-direction flag is in the item index: items [0, n) are (f1, f2),
// items [n, 2n) are (f2, f1).
__global__ void __launch_bounds__(256) k_adjoint(const AdjParams p) {
  extern __shared__ __align__(16) double s_coef[];   // [nb][2]: g/W, -g xi/W of a bin side by side (one 16-byte load)
  for (int k = threadIdx.x; k < 2 * p.nb; k += blockDim.x) s_coef[k] = p.coef[(k & 1) * p.nb + (k >> 1)];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = gw; t < 2 * p.n_items; t += nw) {
    const bool rev = t >= p.n_items;
    const int64_t k = rev ? t - p.n_items : t;
    const int fa = rev ? p.f2[k] : p.f1[k];
    const int fb = rev ? p.f1[k] : p.f2[k];
    const int L1 = p.len[fa], L2 = p.len[fb];
    if (L1 <= 0 || L2 <= 0) continue;
    const int64_t a = p.pstart[fa], b = p.pstart[fb];
    double c = lya_cos12(p.ux[fa], p.uy[fa], p.uz[fa], p.ux[fb], p.uy[fb], p.uz[fb], p.cos_variant);
    c = fmin(1.0, fmax(-1.0, c));
    const double ch = __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(1.0, c)));
    const double sh = __dsqrt_rn(__dmul_rn(0.5, __dsub_rn(1.0, c)));
    const bool srt = p.sorted[fa] && p.sorted[fb];
    const double rp_reach = ch > 0.0 ? ((double)p.np + 1e-3) / (ch * p.binner_rp) : 1e300;
    const double rt_reach = sh > 0.0 ? ((double)p.nt + 1e-3) / (sh * p.binner_rt) : 1e300;
    const double* __restrict__ D2 = p.dc + b;
    const double* __restrict__ W2 = p.w + b;
    const double* __restrict__ DW2 = p.dw + b;
    for (int i0 = 0; i0 < L1; i0 += 32) {
      const int i = i0 + lane;
      double gdw = 0.0, gw_ = 0.0;
      if (i < L1) {
        const double d1 = p.dc[a + i];
        int jlo = 0, jhi = L2;
        if (srt) {
          const double margin = 1e-6 * fabs(d1) + 1e-6;
          const double tlo = d1 - rp_reach - margin;
          const double thi = fmin(d1 + rp_reach, rt_reach - d1) + margin;
          int x = 0, y = L2;
          while (x < y) { const int m = (x + y) >> 1; if (D2[m] > tlo) y = m; else x = m + 1; }
          jlo = x;
          y = L2;
          while (x < y) { const int m = (x + y) >> 1; if (D2[m] < thi) x = m + 1; else y = m; }
          jhi = x;
        }
        // bin of (d1, d2) with the reference FP64 formula, -1 out of range
        auto pbin = [&](double d2) {
          const double rp = __dmul_rn(fabs(__dsub_rn(d1, d2)), ch);
          const double rt = __dmul_rn(__dadd_rn(d1, d2), sh);
          const double fp = floor(__dmul_rn(rp, p.binner_rp));
          const double ft = floor(__dmul_rn(rt, p.binner_rt));
          return (fp >= 0.0 && fp < (double)p.np && ft >= 0.0 && ft < (double)p.nt) ? (int)fp * p.nt + (int)ft : -1;
        };
        // four partners at a time: independent bin chains, then the sums in partner order
        int j = jlo;
        for (; j + 4 <= jhi; j += 4) {
          int bin[4];
          double dwj[4], wj[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            bin[u] = pbin(D2[j + u]);
            dwj[u] = DW2[j + u];
            wj[u] = W2[j + u];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (bin[u] >= 0) {
              const double2 cc = reinterpret_cast<const double2*>(s_coef)[bin[u]];
              gdw = __fma_rn(cc.x, dwj[u], gdw);
              gw_ = __fma_rn(cc.y, wj[u], gw_);
            }
          }
        }
        for (; j < jhi; ++j) {
          const int bn = pbin(D2[j]);
          if (bn >= 0) {
            const double2 cc = reinterpret_cast<const double2*>(s_coef)[bn];
            gdw = __fma_rn(cc.x, DW2[j], gdw);
            gw_ = __fma_rn(cc.y, W2[j], gw_);
          }
        }
        if (gdw != 0.0) atomicAdd(&p.g_dw[a + i], gdw);
        if (gw_ != 0.0) atomicAdd(&p.g_w[a + i], gw_);
      }
    }
  }
}

__global__ void k_unpad(int64_t n, const int64_t* __restrict__ start, const int64_t* __restrict__ pstart,
                        const double* __restrict__ src, double* __restrict__ dst) {
  for (int64_t f = blockIdx.x; f < n; f += gridDim.x) {
    const int64_t s = start[f], L = start[f + 1] - s, d = pstart[f];
    for (int64_t k = threadIdx.x; k < L; k += blockDim.x) dst[s + k] = src[d + k];
  }
}

}  // namespace

// Scratch of the adjoint, kept in the context between calls (grown, never shrunk).
static cudaError_t adjoint_reserve(lya_ctx* ctx, int nb, int64_t n, int64_t npad, int64_t npix) {
  AdjScratch& S = ctx->adj;
  if (S.g && S.nb >= nb && S.n >= n && S.npad >= npad && S.npix >= npix) return cudaSuccess;
  lya_free(S.g); lya_free(S.coef); lya_free(S.gdw); lya_free(S.gw); lya_free(S.out); lya_free(S.start);
  S = AdjScratch{};
  cudaError_t e = lya_alloc(&S.g, nb);
  if (e == cudaSuccess) e = lya_alloc(&S.coef, 2 * (size_t)nb);
  if (e == cudaSuccess) e = lya_alloc(&S.gdw, npad);
  if (e == cudaSuccess) e = lya_alloc(&S.gw, npad);
  if (e == cudaSuccess) e = lya_alloc(&S.out, npix);
  if (e == cudaSuccess) e = lya_alloc(&S.start, n + 1);
  if (e != cudaSuccess) {
    lya_free(S.g); lya_free(S.coef); lya_free(S.gdw); lya_free(S.gw); lya_free(S.out); lya_free(S.start);
    S = AdjScratch{};
    return e;
  }
  S.nb = nb; S.n = n; S.npad = npad; S.npix = npix;
  return cudaSuccess;
}

int lya_adjoint_launch(lya_ctx* ctx, const double* g, double* grad_dw, double* grad_w, int device_ptrs) {
  const int nb = ctx->np * ctx->nt;
  const int64_t n = ctx->cat.n;
  const int64_t npad = ctx->cat.npad, npix = ctx->cat.npix;
  cudaStream_t s = ctx->stream;
  cudaError_t e = adjoint_reserve(ctx, nb, n, npad, npix);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_adjoint: allocation failed");
  AdjScratch& S = ctx->adj;
  double *d_g = S.g, *coef = S.coef, *gdw = S.gdw, *gw = S.gw, *out = S.out;
  int64_t* d_start = S.start;
  e = cudaMemcpyAsync(d_g, g, sizeof(double) * nb, (device_ptrs & 2) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                      s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_start, ctx->h_start.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(gdw, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(gw, 0, sizeof(double) * npad, s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
  if (e == cudaSuccess) {
    k_coef<<<(nb + 255) / 256, 256, 0, s>>>(ctx->hist_slots, nb, ctx->hist, d_g, coef);
    ctx->launches++;
    AdjParams p;
    p.dc = ctx->cat.dc; p.w = ctx->cat.w; p.dw = ctx->cat.dw; p.pstart = ctx->cat.pstart; p.len = ctx->cat.len;
    p.sorted = ctx->cat.sorted; p.ux = ctx->cat.ux; p.uy = ctx->cat.uy; p.uz = ctx->cat.uz;
    p.f1 = ctx->wq.f1; p.f2 = ctx->wq.f2; p.n_items = ctx->wq.n_pairs;
    p.binner_rp = (double)ctx->np / ctx->rpmax; p.binner_rt = (double)ctx->nt / ctx->rtmax;
    p.np = ctx->np; p.nt = ctx->nt; p.nb = nb; p.cos_variant = ctx->cos_variant;
    p.coef = coef; p.g_dw = gdw; p.g_w = gw;
    const size_t smem = sizeof(double) * 2 * nb;
    e = cudaFuncSetAttribute(k_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && p.n_items > 0) {
      k_adjoint<<<ctx->num_sms * 4, 256, smem, s>>>(p);
      ctx->launches++;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
  if (e == cudaSuccess && n > 0) {
    const int blocks = (int)std::min<int64_t>(n, (int64_t)ctx->num_sms * 16);
    if (device_ptrs & 1) {
      if (grad_dw) { k_unpad<<<blocks, 128, 0, s>>>(n, d_start, ctx->cat.pstart, gdw, grad_dw); ctx->launches++; }
      if (grad_w) { k_unpad<<<blocks, 128, 0, s>>>(n, d_start, ctx->cat.pstart, gw, grad_w); ctx->launches++; }
    } else {
      k_unpad<<<blocks, 128, 0, s>>>(n, d_start, ctx->cat.pstart, gdw, out);
      ctx->launches++;
      if (grad_dw) e = cudaMemcpyAsync(grad_dw, out, sizeof(double) * npix, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      k_unpad<<<blocks, 128, 0, s>>>(n, d_start, ctx->cat.pstart, gw, out);
      ctx->launches++;
      if (e == cudaSuccess && grad_w) e = cudaMemcpyAsync(grad_w, out, sizeof(double) * npix, cudaMemcpyDeviceToHost, s);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_corr_adjoint: %s", cudaGetErrorString(e));
  ctx->last.adjoint_ms = ms;
  return LYA_OK;
}

extern "C" int lya_corr_totals(lya_ctx* ctx, double* W, double* DW, int32_t device_ptrs) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_totals: ctx is NULL");
  if (!W || !DW) return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_totals: NULL output");
  if (!ctx->have_result) return lya_fail(ctx, LYA_ERR_STATE, "lya_corr_totals: run lya_corr_run first");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nb = ctx->np * ctx->nt;
  cudaStream_t s = ctx->stream;
  if (device_ptrs) {
    k_totals<<<(nb + 255) / 256, 256, 0, s>>>(ctx->hist_slots, nb, ctx->hist, W, DW);
    ctx->launches++;
    LYA_CHECK_CUDA(ctx, cudaGetLastError());
    LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    return LYA_OK;
  }
  cudaError_t e = adjoint_reserve(ctx, nb, ctx->cat.n, ctx->cat.npad, ctx->cat.npix);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_totals: allocation failed");
  double* t = ctx->adj.coef;   // [2][nb]
  k_totals<<<(nb + 255) / 256, 256, 0, s>>>(ctx->hist_slots, nb, ctx->hist, t, t + nb);
  ctx->launches++;
  LYA_CHECK_CUDA(ctx, cudaGetLastError());
  LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(W, t, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
  LYA_CHECK_CUDA(ctx, cudaMemcpyAsync(DW, t + nb, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  return LYA_OK;
}

extern "C" int lya_corr_adjoint(lya_ctx* ctx, const double* g, double* grad_dw, double* grad_w, int32_t device_ptrs) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_adjoint: ctx is NULL");
  if (!g) return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_adjoint: g is NULL");
  if (!ctx->have_result) return lya_fail(ctx, LYA_ERR_STATE, "lya_corr_adjoint: run lya_corr_run first");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  return lya_adjoint_launch(ctx, g, grad_dw, grad_w, device_ptrs);
}
