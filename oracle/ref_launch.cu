// Launcher of the reference's own CUDA kernels.  TEST INFRASTRUCTURE ONLY.
//
// The reference compiles cuda_kernels.cpp at run time with PyCUDA's
// SourceModule (nvcc defaults, source wrapped in extern "C"); PyCUDA is not
// available, so oracle/Makefile compiles the same file from the reference tree
// with nvcc and this launcher drives pair_correlation exactly as
// correlation_procedures_pycuda.two_point_per_pixel does
// (correlation_procedures_pycuda.py:141-166): one launch per first forest,
// grid (len1, 1, 1), block (1, 16, 16), a synchronize after each launch, FP64
// histograms accumulated with global atomics.
//
// The reference kernel has two input hazards that write outside its
// histograms: cos12 > 1 (sqrt of a negative number, cuda_kernels.cpp:132-134)
// and dc < 0 (negative rt bin, :150-153).  The launcher refuses such inputs
// instead of launching.
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
