// Launcher of the reference's own CUDA kernels.  TEST INFRASTRUCTURE ONLY.
//
// The reference compiles cuda_kernels.cpp at run time with PyCUDA's
// SourceModule (nvcc defaults, source wrapped in extern "C"); PyCUDA is not
// available, so oracle/Makefile compiles the same file from the reference tree
// with nvcc and this launcher drives
//  * pair_correlation exactly as correlation_procedures_pycuda.two_point_per_pixel
//    does (correlation_procedures_pycuda.py:141-166): one launch per first
//    forest, grid (len1, 1, 1), block (1, 16, 16), a synchronize after each
//    launch, FP64 histograms accumulated with global atomics;
//  * precompute_distances, compute_etas, order_active and compute_d exactly as
//    distortion_procedures.distortion_per_pixel does
//    (distortion_procedures_pycuda.py:202-279): FP32 padded inputs, per first
//    forest the eight eta memsets, index_j = 0, ActiveBs = 0,
//    ActiveBs_index = -1, then the four launches with block (8, 32, 4) /
//    (32, 32, 1) and grids from the first forest's length, max_lenght and the
//    neighbour count (parameters.py:54-56); D and W_B accumulate over the
//    pixel's first forests and are cleared once per call.
//
// The reference kernels have input hazards that read or write outside their
// buffers: cos12 > 1 (sqrt of a negative number, cuda_kernels.cpp:132-134,
// :73-74), dc < 0 (negative bins pass the upper-edge-only tests, :150-153,
// :193, :256), forests longer than max_lenght, more neighbours than the scratch
// holds (:64, :191), and compute_d's read of ActiveBs_index one element past a
// full row before its bound test (:259).  The launcher refuses the first three
// instead of launching, sizes the scratch for the largest neighbour list, and
// gives ActiveBs_index one padding row of -1.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <vector>

extern "C" {
#include REF_KERNELS_SOURCE
}

static int fail(const char* what, cudaError_t e) {
  fprintf(stderr, "ref_launch: %s: %s\n", what, cudaGetErrorString(e));
  return 2;
}

#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return fail(#call, e_); \
  } while (0)

static double cos_variant(double x1, double y1, double z1, double x2, double y2, double z2, int v) {
  if (v == 0) return fma(z1, z2, fma(x1, x2, y1 * y2));
  if (v == 1) return fma(z1, z2, fma(y1, y2, x1 * x2));
  double a = x1 * x2, b = y1 * y2, c = z1 * z2;
  return (a + b) + c;
}

// Histograms of one owner pixel: first forests f1_list[k] with neighbours
// nbr[nbr_off[k] .. nbr_off[k+1]).  Forests are padded to max_len pixels in
// dc/we/dw ([n_forest * max_len]).  Returns 0, 1 (unsafe input), 2 (CUDA).
extern "C" int ref_corr_pixel(int n_forest, int max_len, const double* dc, const double* we, const double* dw,
                              const int* len, const double* x, const double* y, const double* z, int n_f1,
                              const int* f1_list, const int64_t* nbr_off, const int* nbr, double rpmax,
                              double rtmax, int np, int nt, double* w_hist, double* dw_hist) {
  for (int k = 0; k < n_f1; ++k) {
    const int f1 = f1_list[k];
    for (int64_t q = nbr_off[k]; q < nbr_off[k + 1]; ++q) {
      const int f2 = nbr[q];
      for (int v = 0; v < 3; ++v)
        if (cos_variant(x[f1], y[f1], z[f1], x[f2], y[f2], z[f2], v) > 1.0) return 1;
    }
  }
  for (int64_t i = 0; i < (int64_t)n_forest * max_len; ++i)
    if (!(dc[i] >= 0.0)) return 1;
  const size_t big = sizeof(double) * (size_t)n_forest * max_len;
  const size_t small = sizeof(double) * (size_t)n_forest;
  const size_t hist = sizeof(double) * (size_t)np * nt;
  double *d_dc, *d_we, *d_dw, *d_x, *d_y, *d_z, *d_w_hist, *d_dw_hist, *d_rmax;
  int *d_base, *d_idx, *d_sizes, *d_numpix;
  int maxn = 1;
  for (int k = 0; k < n_f1; ++k) maxn = (int)fmax((double)maxn, (double)(nbr_off[k + 1] - nbr_off[k]));
  CK(cudaMalloc(&d_dc, big)); CK(cudaMalloc(&d_we, big)); CK(cudaMalloc(&d_dw, big));
  CK(cudaMalloc(&d_x, small)); CK(cudaMalloc(&d_y, small)); CK(cudaMalloc(&d_z, small));
  CK(cudaMalloc(&d_w_hist, hist)); CK(cudaMalloc(&d_dw_hist, hist)); CK(cudaMalloc(&d_rmax, 2 * sizeof(double)));
  CK(cudaMalloc(&d_base, 3 * sizeof(int))); CK(cudaMalloc(&d_numpix, 2 * sizeof(int)));
  CK(cudaMalloc(&d_idx, maxn * sizeof(int))); CK(cudaMalloc(&d_sizes, maxn * sizeof(int)));
  CK(cudaMemcpy(d_dc, dc, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_we, we, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_dw, dw, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_x, x, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_y, y, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_z, z, small, cudaMemcpyHostToDevice));
  CK(cudaMemset(d_w_hist, 0, hist));
  CK(cudaMemset(d_dw_hist, 0, hist));
  const double rmax[2] = {rpmax, rtmax};
  const int numpix[2] = {np, nt};
  CK(cudaMemcpy(d_rmax, rmax, sizeof(rmax), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_numpix, numpix, sizeof(numpix), cudaMemcpyHostToDevice));
  std::vector<int> idx, sizes;
  for (int k = 0; k < n_f1; ++k) {
    const int f1 = f1_list[k];
    const int nn = (int)(nbr_off[k + 1] - nbr_off[k]);
    if (nn == 0) continue;   // correlation_procedures_pycuda.py:145-147
    idx.assign(nbr + nbr_off[k], nbr + nbr_off[k + 1]);
    sizes.resize(nn);
    for (int q = 0; q < nn; ++q) sizes[q] = len[idx[q]];
    const int base[3] = {f1, len[f1], nn};
    CK(cudaMemcpy(d_base, base, sizeof(base), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_idx, idx.data(), nn * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_sizes, sizes.data(), nn * sizeof(int), cudaMemcpyHostToDevice));
    // rx, ry, rz are unused by the kernel; the reference passes its own copies
    pair_correlation<<<dim3(len[f1], 1, 1), dim3(1, 16, 16)>>>(d_base, d_idx, d_sizes, d_numpix, max_len, d_rmax,
                                                                d_w_hist, d_dw_hist, d_dc, d_dc, d_dc, d_dc, d_we,
                                                                d_dw, d_x, d_y, d_z);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
  CK(cudaMemcpy(w_hist, d_w_hist, hist, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(dw_hist, d_dw_hist, hist, cudaMemcpyDeviceToHost));
  cudaFree(d_dc); cudaFree(d_we); cudaFree(d_dw); cudaFree(d_x); cudaFree(d_y); cudaFree(d_z);
  cudaFree(d_w_hist); cudaFree(d_dw_hist); cudaFree(d_rmax); cudaFree(d_base); cudaFree(d_numpix);
  cudaFree(d_idx); cudaFree(d_sizes);
  return 0;
}

// ------------------------------------------------------------------ distortion
static bool safe_fp32_cos(float x1, float y1, float z1, float x2, float y2, float z2) {
  const float c0 = fmaf(z1, z2, fmaf(x1, x2, y1 * y2));
  const float c1 = fmaf(z1, z2, fmaf(y1, y2, x1 * x2));
  const float c2 = (x1 * x2 + y1 * y2) + z1 * z2;
  return c0 <= 1.0f && c1 <= 1.0f && c2 <= 1.0f && c0 >= -1.0f && c1 >= -1.0f && c2 >= -1.0f;
}

struct DistBuffers {
  float *dc = 0, *rxyz = 0, *we = 0, *dl = 0, *x = 0, *y = 0, *z = 0, *odl2 = 0, *omega = 0, *binner = 0;
  float *e12 = 0, *e21 = 0, *e13 = 0, *e31 = 0, *e22 = 0, *e23 = 0, *e32 = 0, *e33 = 0, *wb = 0, *d = 0;
  float *x12 = 0, *y12 = 0, *z12 = 0, *r12 = 0;
  int *bin_rp = 0, *bin_rt = 0, *numpix = 0, *base = 0, *idx = 0, *sizes = 0, *active_index = 0, *index_j = 0;
  bool* active = 0;
  ~DistBuffers() {
    void* all[] = {dc, rxyz, we, dl, x, y, z, odl2, omega, binner, e12, e21, e13, e31, e22, e23, e32, e33, wb, d,
                   x12, y12, z12, r12, bin_rp, bin_rt, numpix, base, idx, sizes, active_index, index_j, active};
    for (void* p : all)
      if (p) cudaFree(p);
  }
};

// Checks shared by the distortion entry points.  Returns 0 when the reference
// kernels stay inside their buffers for these inputs, 1 otherwise.
static int dist_inputs_safe(int n_forest, int max_len, const float* dc, const int* len, const float* x,
                            const float* y, const float* z, int n_f1, const int* f1_list, const int64_t* nbr_off,
                            const int* nbr, int* max_nn) {
  if (n_forest <= 0 || max_len <= 0) return 1;
  for (int f = 0; f < n_forest; ++f)
    if (len[f] < 0 || len[f] > max_len) return 1;
  for (int64_t i = 0; i < (int64_t)n_forest * max_len; ++i)
    if (!(dc[i] >= 0.0f) || !(dc[i] < 1.0e7f)) return 1;
  int mx = 1;
  for (int k = 0; k < n_f1; ++k) {
    const int f1 = f1_list[k];
    if (f1 < 0 || f1 >= n_forest || len[f1] == 0) return 1;
    const int64_t nn = nbr_off[k + 1] - nbr_off[k];
    if (nn < 0 || nn > 100000) return 1;
    if (nn > mx) mx = (int)nn;
    for (int64_t q = nbr_off[k]; q < nbr_off[k + 1]; ++q) {
      const int f2 = nbr[q];
      if (f2 < 0 || f2 >= n_forest) return 1;
      if (!safe_fp32_cos(x[f1], y[f1], z[f1], x[f2], y[f2], z[f2])) return 1;
    }
  }
  *max_nn = mx;
  return 0;
}

static int dist_alloc(DistBuffers& B, int n_forest, int max_len, int nn_cap, int nb, const float* dc,
                      const float* we, const float* dl, const float* x, const float* y, const float* z,
                      const float* omega, const float* odl2, float binner_rp, float binner_rt, int np, int nt) {
  const size_t big = sizeof(float) * (size_t)n_forest * max_len;
  const size_t small = sizeof(float) * (size_t)n_forest;
  const size_t eta = sizeof(float) * (size_t)nn_cap * nb * max_len;
  const size_t eta_small = sizeof(float) * (size_t)nn_cap * nb;
  const size_t aux = sizeof(float) * (size_t)max_len * max_len * nn_cap;
  CK(cudaMalloc(&B.dc, big)); CK(cudaMalloc(&B.rxyz, big)); CK(cudaMalloc(&B.we, big)); CK(cudaMalloc(&B.dl, big));
  CK(cudaMalloc(&B.x, small)); CK(cudaMalloc(&B.y, small)); CK(cudaMalloc(&B.z, small));
  CK(cudaMalloc(&B.odl2, small)); CK(cudaMalloc(&B.omega, small)); CK(cudaMalloc(&B.binner, 2 * sizeof(float)));
  CK(cudaMalloc(&B.e12, eta)); CK(cudaMalloc(&B.e21, eta)); CK(cudaMalloc(&B.e13, eta)); CK(cudaMalloc(&B.e31, eta));
  CK(cudaMalloc(&B.e22, eta_small)); CK(cudaMalloc(&B.e23, eta_small)); CK(cudaMalloc(&B.e32, eta_small));
  CK(cudaMalloc(&B.e33, eta_small));
  CK(cudaMalloc(&B.wb, sizeof(float) * nb)); CK(cudaMalloc(&B.d, sizeof(float) * (size_t)nb * nb));
  CK(cudaMalloc(&B.x12, aux)); CK(cudaMalloc(&B.y12, aux)); CK(cudaMalloc(&B.z12, aux)); CK(cudaMalloc(&B.r12, aux));
  CK(cudaMalloc(&B.bin_rp, aux)); CK(cudaMalloc(&B.bin_rt, aux));
  CK(cudaMalloc(&B.numpix, 2 * sizeof(int))); CK(cudaMalloc(&B.base, 3 * sizeof(int)));
  CK(cudaMalloc(&B.idx, sizeof(int) * nn_cap)); CK(cudaMalloc(&B.sizes, sizeof(int) * nn_cap));
  // one padding row: compute_d reads ActiveBs_index[f2*tot_pix + tot_pix] before its bound test
  CK(cudaMalloc(&B.active_index, sizeof(int) * (size_t)(nn_cap + 1) * nb));
  CK(cudaMalloc(&B.index_j, sizeof(int) * nn_cap));
  CK(cudaMalloc(&B.active, sizeof(bool) * (size_t)nn_cap * nb));
  CK(cudaMemcpy(B.dc, dc, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.rxyz, dc, big, cudaMemcpyHostToDevice));   // rx/ry/rz feed only the unused x12..r12
  CK(cudaMemcpy(B.we, we, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.dl, dl, big, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.x, x, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.y, y, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.z, z, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.omega, omega, small, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.odl2, odl2, small, cudaMemcpyHostToDevice));
  const float binner[2] = {binner_rp, binner_rt};
  const int numpix[2] = {np, nt};
  CK(cudaMemcpy(B.binner, binner, sizeof(binner), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.numpix, numpix, sizeof(numpix), cudaMemcpyHostToDevice));
  CK(cudaMemset(B.d, 0, sizeof(float) * (size_t)nb * nb));   // distortion_procedures_pycuda.py:204-205
  CK(cudaMemset(B.wb, 0, sizeof(float) * nb));
  return 0;
}

// One first forest: the memsets and the four launches of
// distortion_procedures_pycuda.py:209-274.  nn > 0.
static int dist_one(DistBuffers& B, int max_len, int nn_cap, int nb, int f1, int len1, const int* idx, const int* len,
                    int nn, bool all_kernels) {
  const size_t eta = sizeof(float) * (size_t)nn_cap * nb * max_len;
  const size_t eta_small = sizeof(float) * (size_t)nn_cap * nb;
  CK(cudaMemset(B.e12, 0, eta)); CK(cudaMemset(B.e13, 0, eta)); CK(cudaMemset(B.e21, 0, eta));
  CK(cudaMemset(B.e31, 0, eta));
  CK(cudaMemset(B.e22, 0, eta_small)); CK(cudaMemset(B.e23, 0, eta_small)); CK(cudaMemset(B.e32, 0, eta_small));
  CK(cudaMemset(B.e33, 0, eta_small));
  CK(cudaMemset(B.index_j, 0, sizeof(int) * nn_cap));
  CK(cudaMemset(B.active, 0, sizeof(bool) * (size_t)nn_cap * nb));
  CK(cudaMemset(B.active_index, 0xff, sizeof(int) * (size_t)(nn_cap + 1) * nb));
  std::vector<int> sizes(nn);
  for (int q = 0; q < nn; ++q) sizes[q] = len[idx[q]];
  const int base[3] = {f1, len1, nn};
  CK(cudaMemcpy(B.base, base, sizeof(base), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.idx, idx, nn * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.sizes, sizes.data(), nn * sizeof(int), cudaMemcpyHostToDevice));
  const dim3 tpb(8, 32, 4), tpb2(32, 32, 1);
  const dim3 grid((len1 + 7) / 8, (max_len + 31) / 32, (nn + 3) / 4);
  const dim3 grid2((nb + 31) / 32, (nn + 31) / 32, 1);
  precompute_distances<<<grid, tpb>>>(max_len, B.base, B.idx, B.sizes, B.binner, B.rxyz, B.rxyz, B.rxyz, B.x, B.y,
                                      B.z, B.dc, B.x12, B.y12, B.z12, B.r12, B.bin_rp, B.bin_rt);
  CK(cudaGetLastError());
  if (all_kernels) {
    compute_etas<<<grid, tpb>>>(max_len, B.numpix, B.base, B.idx, B.sizes, B.we, B.dl, B.bin_rp, B.bin_rt, B.odl2,
                                B.omega, B.active, B.e12, B.e21, B.e22, B.e13, B.e31, B.e23, B.e32, B.e33, B.wb);
    CK(cudaGetLastError());
    order_active<<<grid2, tpb2>>>(B.active, B.active_index, B.numpix, B.base, B.index_j);
    CK(cudaGetLastError());
    compute_d<<<grid, tpb>>>(max_len, B.numpix, B.base, B.idx, B.sizes, B.we, B.dl, B.bin_rp, B.bin_rt,
                             B.active_index, B.e12, B.e21, B.e22, B.e13, B.e31, B.e23, B.e32, B.e33, B.d);
    CK(cudaGetLastError());
  }
  CK(cudaDeviceSynchronize());
  return 0;
}

// Distortion numerator D [nb x nb] and bin weights W_B [nb] of one healpix
// pixel: first forests f1_list[k] with (already subsampled) neighbour lists
// nbr[nbr_off[k] .. nbr_off[k+1]).  Inputs are FP32 and padded to max_len
// pixels ([n_forest * max_len]) like the reference's gran_* arrays.  Returns 0,
// 1 (unsafe input) or 2 (CUDA error).
extern "C" int ref_dist_pixel(int n_forest, int max_len, const float* dc, const float* we, const float* dl,
                              const int* len, const float* x, const float* y, const float* z, const float* omega,
                              const float* odl2, int n_f1, const int* f1_list, const int64_t* nbr_off,
                              const int* nbr, float binner_rp, float binner_rt, int np, int nt, float* D,
                              float* WB) {
  int nn_cap = 1;
  if (np <= 0 || nt <= 0 || np * nt > 10000) return 1;
  if (dist_inputs_safe(n_forest, max_len, dc, len, x, y, z, n_f1, f1_list, nbr_off, nbr, &nn_cap)) return 1;
  const int nb = np * nt;
  DistBuffers B;
  int rc = dist_alloc(B, n_forest, max_len, nn_cap, nb, dc, we, dl, x, y, z, omega, odl2, binner_rp, binner_rt, np, nt);
  if (rc) return rc;
  for (int k = 0; k < n_f1; ++k) {
    const int nn = (int)(nbr_off[k + 1] - nbr_off[k]);
    if (nn == 0) continue;   // distortion_procedures_pycuda.py:233-235
    rc = dist_one(B, max_len, nn_cap, nb, f1_list[k], len[f1_list[k]], nbr + nbr_off[k], len, nn, true);
    if (rc) return rc;
  }
  CK(cudaMemcpy(D, B.d, sizeof(float) * (size_t)nb * nb, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(WB, B.wb, sizeof(float) * nb, cudaMemcpyDeviceToHost));
  return 0;
}

// bin_rp and bin_rt that precompute_distances writes for one first forest and
// its neighbour list, laid out [len1][nn][max_len] as the kernel indexes them
// ((i * nn + f2) * max_len + j).  Returns 0, 1 (unsafe input) or 2.
extern "C" int ref_dist_bins(int n_forest, int max_len, const float* dc, const int* len, const float* x,
                             const float* y, const float* z, int f1, int nn, const int* nbr, float binner_rp,
                             float binner_rt, int32_t* bin_rp, int32_t* bin_rt) {
  int nn_cap = 1;
  const int64_t off[2] = {0, nn};
  if (nn <= 0) return 1;
  if (dist_inputs_safe(n_forest, max_len, dc, len, x, y, z, 1, &f1, off, nbr, &nn_cap)) return 1;
  const int nb = 1;
  std::vector<float> zero((size_t)n_forest * max_len, 0.0f), ones(n_forest, 1.0f);
  DistBuffers B;
  int rc = dist_alloc(B, n_forest, max_len, nn_cap, nb, dc, zero.data(), zero.data(), x, y, z, ones.data(),
                      ones.data(), binner_rp, binner_rt, 1, 1);
  if (rc) return rc;
  const size_t aux = sizeof(int32_t) * (size_t)max_len * max_len * nn_cap;
  CK(cudaMemset(B.bin_rp, 0xff, aux));
  CK(cudaMemset(B.bin_rt, 0xff, aux));
  rc = dist_one(B, max_len, nn_cap, nb, f1, len[f1], nbr, len, nn, false);
  if (rc) return rc;
  const size_t n_out = sizeof(int32_t) * (size_t)len[f1] * nn * max_len;
  CK(cudaMemcpy(bin_rp, B.bin_rp, n_out, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(bin_rt, B.bin_rt, n_out, cudaMemcpyDeviceToHost));
  return 0;
}

// ------------------------------------------------------------------ timing
// The reference's pair_correlation driven exactly as ref_corr_pixel drives it
// (per first forest: three small copies, one launch, a synchronize), with the
// padded catalogue uploaded once before the timed loop.  *ms receives the
// device time of the loop (CUDA events around it), w_hist/dw_hist the
// histograms.  Returns 0, 1 (unsafe input) or 2.
extern "C" int ref_corr_timed(int n_forest, int max_len, const double* dc, const double* we, const double* dw,
                              const int* len, const double* x, const double* y, const double* z, int n_f1,
                              const int* f1_list, const int64_t* nbr_off, const int* nbr, double rpmax, double rtmax,
                              int np, int nt, double* w_hist, double* dw_hist, double* ms) {
  for (int k = 0; k < n_f1; ++k) {
    const int f1 = f1_list[k];
    if (f1 < 0 || f1 >= n_forest || len[f1] < 0 || len[f1] > max_len) return 1;
    for (int64_t q = nbr_off[k]; q < nbr_off[k + 1]; ++q) {
      const int f2 = nbr[q];
      if (f2 < 0 || f2 >= n_forest || len[f2] < 0 || len[f2] > max_len) return 1;
      for (int v = 0; v < 3; ++v)
        if (cos_variant(x[f1], y[f1], z[f1], x[f2], y[f2], z[f2], v) > 1.0) return 1;
    }
  }
  for (int64_t i = 0; i < (int64_t)n_forest * max_len; ++i)
    if (!(dc[i] >= 0.0)) return 1;
  const size_t big = sizeof(double) * (size_t)n_forest * max_len;
  const size_t small = sizeof(double) * (size_t)n_forest;
  const size_t hist = sizeof(double) * (size_t)np * nt;
  int maxn = 1;
  for (int k = 0; k < n_f1; ++k) maxn = (int)fmax((double)maxn, (double)(nbr_off[k + 1] - nbr_off[k]));
  double *d_dc = 0, *d_we = 0, *d_dw = 0, *d_x = 0, *d_y = 0, *d_z = 0, *d_w_hist = 0, *d_dw_hist = 0, *d_rmax = 0;
  int *d_base = 0, *d_idx = 0, *d_sizes = 0, *d_numpix = 0;
  cudaEvent_t e0 = 0, e1 = 0;
  int rc = 0;
  do {
#define CKB(call) { cudaError_t e_ = (call); if (e_ != cudaSuccess) { rc = fail(#call, e_); break; } }
    CKB(cudaMalloc(&d_dc, big)); CKB(cudaMalloc(&d_we, big)); CKB(cudaMalloc(&d_dw, big));
    CKB(cudaMalloc(&d_x, small)); CKB(cudaMalloc(&d_y, small)); CKB(cudaMalloc(&d_z, small));
    CKB(cudaMalloc(&d_w_hist, hist)); CKB(cudaMalloc(&d_dw_hist, hist)); CKB(cudaMalloc(&d_rmax, 2 * sizeof(double)));
    CKB(cudaMalloc(&d_base, 3 * sizeof(int))); CKB(cudaMalloc(&d_numpix, 2 * sizeof(int)));
    CKB(cudaMalloc(&d_idx, maxn * sizeof(int))); CKB(cudaMalloc(&d_sizes, maxn * sizeof(int)));
    CKB(cudaMemcpy(d_dc, dc, big, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_we, we, big, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_dw, dw, big, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_x, x, small, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_y, y, small, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_z, z, small, cudaMemcpyHostToDevice));
    CKB(cudaMemset(d_w_hist, 0, hist));
    CKB(cudaMemset(d_dw_hist, 0, hist));
    const double rmax[2] = {rpmax, rtmax};
    const int numpix[2] = {np, nt};
    CKB(cudaMemcpy(d_rmax, rmax, sizeof(rmax), cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_numpix, numpix, sizeof(numpix), cudaMemcpyHostToDevice));
    CKB(cudaEventCreate(&e0)); CKB(cudaEventCreate(&e1));
    std::vector<int> sizes;
    CKB(cudaDeviceSynchronize());
    CKB(cudaEventRecord(e0));
    for (int k = 0; k < n_f1 && rc == 0; ++k) {
      const int f1 = f1_list[k];
      const int nn = (int)(nbr_off[k + 1] - nbr_off[k]);
      if (nn == 0 || len[f1] == 0) continue;
      sizes.resize(nn);
      for (int q = 0; q < nn; ++q) sizes[q] = len[nbr[nbr_off[k] + q]];
      const int base[3] = {f1, len[f1], nn};
      CKB(cudaMemcpy(d_base, base, sizeof(base), cudaMemcpyHostToDevice));
      CKB(cudaMemcpy(d_idx, nbr + nbr_off[k], nn * sizeof(int), cudaMemcpyHostToDevice));
      CKB(cudaMemcpy(d_sizes, sizes.data(), nn * sizeof(int), cudaMemcpyHostToDevice));
      pair_correlation<<<dim3(len[f1], 1, 1), dim3(1, 16, 16)>>>(d_base, d_idx, d_sizes, d_numpix, max_len, d_rmax,
                                                                  d_w_hist, d_dw_hist, d_dc, d_dc, d_dc, d_dc, d_we,
                                                                  d_dw, d_x, d_y, d_z);
      CKB(cudaGetLastError());
      CKB(cudaDeviceSynchronize());
    }
    if (rc) break;
    CKB(cudaEventRecord(e1));
    CKB(cudaEventSynchronize(e1));
    float f = 0.f;
    CKB(cudaEventElapsedTime(&f, e0, e1));
    *ms = f;
    CKB(cudaMemcpy(w_hist, d_w_hist, hist, cudaMemcpyDeviceToHost));
    CKB(cudaMemcpy(dw_hist, d_dw_hist, hist, cudaMemcpyDeviceToHost));
#undef CKB
  } while (0);
  void* all[] = {d_dc, d_we, d_dw, d_x, d_y, d_z, d_w_hist, d_dw_hist, d_rmax, d_base, d_idx, d_sizes, d_numpix};
  for (void* p : all)
    if (p) cudaFree(p);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return rc;
}
