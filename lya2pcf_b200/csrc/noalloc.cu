// Histogram of one owner pixel with no device allocation.
//
// Some callers cannot allocate device memory: a host program whose device
// memory is handed out by another framework's caching allocator (a cudaMalloc
// of its own would fragment or exceed that allocator's pool), a service that
// runs under a fixed device-memory budget, or code that must not add
// allocation calls to a sequence it records for later replay.  They cannot use
// lya_upload_forests / lya_corr_run, which allocate the packed catalogue, the
// work queue and the per-pixel outputs.  lya_corr_pixel_noalloc takes the
// catalogue, the forest-pair list and the output histograms in the caller's
// device memory and keeps its only scratch -- the compensated FP64
// accumulators, LYA_NQ x 2 x 4096 doubles = 320 KB -- in a file-scope
// __device__ array, so it calls no cudaMalloc, cudaFree or allocating library
// routine.  Consequences of the shared array:
//   * every GPU that loads the library holds the 320 KB until the process exits;
//   * the first call on a device does that device's set-up with the device
//     current: it looks the array's device address up (cudaGetSymbolAddress),
//     raises the kernel's dynamic shared-memory limit to what 4096 bins need,
//     loads both kernels and reads the SM count; later calls make none of
//     these driver calls.  Make that first call before any stream capture;
//   * the call selects the device itself (cudaSetDevice on the library's own,
//     statically linked, CUDA runtime);
//   * every call clears the part of the array it uses, but all calls share it:
//     calls that overlap on the GPU (different streams or threads without
//     ordering) race on it and give wrong sums.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "lya_internal.cuh"

#define LYA_NOALLOC_MAX_BINS 4096

namespace {

// (hi, lo) FP64 accumulators of the LYA_NQ quantities: [LYA_NQ][2][bins].
// Shared by every call on a device; the contents of the last call stay there
// until the next call clears them.
static __device__ __align__(256) double g_noalloc_acc[LYA_NQ * 2 * LYA_NOALLOC_MAX_BINS];

__device__ __forceinline__ void add_comp(double* hi, double* lo, double v) {
  const double old = atomicAdd(hi, v);
  const double s = old + v;
  const double bb = s - old;
  const double err = (old - (s - bb)) + (v - bb);
  if (err != 0.0) atomicAdd(lo, err);
}

struct NoAllocParams {
  const double* dc; const double* w; const double* dw; const double* z;
  const int64_t* start;
  const double* ux; const double* uy; const double* uz;
  const int32_t* f1; const int32_t* f2;
  int64_t n_pairs;
  double binner_rp, binner_rt;
  int np, nt, nb;
  double* acc;                       // device address of g_noalloc_acc
  unsigned long long* counts;        // caller's output
};

// Every pixel pair of every listed forest pair, FP64 reference formula; one
// warp per forest pair, shared-memory FP64 histogram per CTA, flushed once.
__global__ void __launch_bounds__(256) k_corr_noalloc(const NoAllocParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sq = reinterpret_cast<double*>(smem);                         // [LYA_NQ][nb]
  unsigned long long* sn = reinterpret_cast<unsigned long long*>(sq + LYA_NQ * p.nb);
  for (int k = threadIdx.x; k < LYA_NQ * p.nb; k += blockDim.x) sq[k] = 0.0;
  for (int k = threadIdx.x; k < p.nb; k += blockDim.x) sn[k] = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = gw; t < p.n_pairs; t += nw) {
    const int a = p.f1[t], b = p.f2[t];
    const int64_t s1 = p.start[a], L1 = p.start[a + 1] - s1;
    const int64_t s2 = p.start[b], L2 = p.start[b + 1] - s2;
    double c = lya_cos12(p.ux[a], p.uy[a], p.uz[a], p.ux[b], p.uy[b], p.uz[b], 0);
    c = fmin(1.0, fmax(-1.0, c));
    const double ch = __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(1.0, c)));
    const double sh = __dsqrt_rn(__dmul_rn(0.5, __dsub_rn(1.0, c)));
    for (int64_t i = 0; i < L1; ++i) {
      const double d1 = p.dc[s1 + i], w1 = p.w[s1 + i], dw1 = p.dw[s1 + i], z1 = p.z[s1 + i];
      for (int64_t j = lane; j < L2; j += 32) {
        const double d2 = p.dc[s2 + j];
        const double rp = __dmul_rn(fabs(__dsub_rn(d1, d2)), ch);
        const double rt = __dmul_rn(__dadd_rn(d1, d2), sh);
        const double fp = floor(__dmul_rn(rp, p.binner_rp));
        const double ft = floor(__dmul_rn(rt, p.binner_rt));
        if (fp >= 0.0 && fp < (double)p.np && ft >= 0.0 && ft < (double)p.nt) {
          const int k = (int)fp * p.nt + (int)ft;
          const double w12 = __dmul_rn(w1, p.w[s2 + j]);
          atomicAdd(&sq[0 * p.nb + k], w12);
          atomicAdd(&sq[1 * p.nb + k], __dmul_rn(dw1, p.dw[s2 + j]));
          atomicAdd(&sq[2 * p.nb + k], __dmul_rn(w12, rp));
          atomicAdd(&sq[3 * p.nb + k], __dmul_rn(w12, rt));
          atomicAdd(&sq[4 * p.nb + k], __dmul_rn(w12, __dadd_rn(z1, p.z[s2 + j])));
          atomicAdd(&sn[k], 1ull);
        }
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < LYA_NQ * p.nb; k += blockDim.x) {
    const int q = k / p.nb, bb = k - q * p.nb;
    double v = sq[k];
    if (q == 4) v *= 0.5;
    if (v != 0.0) add_comp(p.acc + (size_t)(q * 2) * p.nb + bb, p.acc + (size_t)(q * 2 + 1) * p.nb + bb, v);
  }
  for (int k = threadIdx.x; k < p.nb; k += blockDim.x)
    if (sn[k]) atomicAdd(&p.counts[k], sn[k]);
}

__global__ void k_noalloc_combine(int nb, const double* __restrict__ acc, double* __restrict__ hist) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < LYA_NQ * nb; k += gridDim.x * blockDim.x) {
    const int q = k / nb, b = k - q * nb;
    hist[k] = acc[(q * 2) * nb + b] + acc[(q * 2 + 1) * nb + b];
  }
}

// Per-device state of the set-up done by the first call on each device.
struct DeviceSetup {
  double* acc;   // device address of g_noalloc_acc on that device
  int sms;       // multiprocessor count
};
std::mutex g_setup_mu;
DeviceSetup g_setup[64] = {};
bool g_ready[64] = {};

// Set-up of `device` (which is current): cudaGetSymbolAddress of the scratch,
// the shared-memory limit for the largest binning, a first touch of both
// kernels (so that no later call loads a kernel, even one that launches only
// the combine step), and the SM count.
cudaError_t setup_device(int device, DeviceSetup* out) {
  DeviceSetup d = {nullptr, 148};
  cudaError_t e = cudaGetSymbolAddress((void**)&d.acc, g_noalloc_acc);
  if (e != cudaSuccess) return e;
  const size_t smem_max = (size_t)LYA_NOALLOC_MAX_BINS * (LYA_NQ * sizeof(double) + sizeof(unsigned long long));
  e = cudaFuncSetAttribute(k_corr_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, k_noalloc_combine);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  *out = d;
  return cudaSuccess;
}

}  // namespace

extern "C" int lya_corr_pixel_noalloc(int device, const double* dc, const double* w, const double* dw,
                                      const double* z, const int64_t* start, const double* ux, const double* uy,
                                      const double* uz, const int32_t* f1, const int32_t* f2, int64_t n_pairs,
                                      double rpmax, double rtmax, int32_t np, int32_t nt, double* hist,
                                      uint64_t* counts, void* stream) {
  if (!(rpmax > 0) || !(rtmax > 0) || np <= 0 || nt <= 0)
    return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_pixel_noalloc: need rpmax, rtmax > 0 and np, nt > 0");
  if ((int64_t)np * nt > LYA_NOALLOC_MAX_BINS)
    return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_pixel_noalloc: np*nt = %lld exceeds the fixed scratch of %d bins",
                    (long long)np * nt, LYA_NOALLOC_MAX_BINS);
  if (n_pairs < 0 || (n_pairs > 0 && (!dc || !w || !dw || !z || !start || !ux || !uy || !uz || !f1 || !f2)) ||
      !hist || !counts)
    return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_pixel_noalloc: NULL device pointer or negative n_pairs");
  if (device < 0 || device >= 64) return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_pixel_noalloc: bad device");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return lya_fail(nullptr, LYA_ERR_CUDA, "lya_corr_pixel_noalloc: %s", cudaGetErrorString(e));
  DeviceSetup dev;
  {
    // set-up once per device, with that device current: the device address of
    // the scratch array (its host-side name is only a stand-in) and the rest
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_ready[device]) {
      e = setup_device(device, &g_setup[device]);
      if (e != cudaSuccess)
        return lya_fail(nullptr, LYA_ERR_CUDA, "lya_corr_pixel_noalloc: set-up of device %d: %s", device,
                        cudaGetErrorString(e));
      g_ready[device] = true;
    }
    dev = g_setup[device];
  }
  double* acc = dev.acc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nb = np * nt;
  e = cudaMemsetAsync(acc, 0, sizeof(double) * LYA_NQ * 2 * (size_t)nb, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, sizeof(uint64_t) * (size_t)nb, s);
  if (e == cudaSuccess && n_pairs > 0) {
    NoAllocParams p;
    p.dc = dc; p.w = w; p.dw = dw; p.z = z; p.start = start; p.ux = ux; p.uy = uy; p.uz = uz; p.f1 = f1; p.f2 = f2;
    p.n_pairs = n_pairs; p.binner_rp = (double)np / rpmax; p.binner_rt = (double)nt / rtmax;
    p.np = np; p.nt = nt; p.nb = nb; p.acc = acc; p.counts = reinterpret_cast<unsigned long long*>(counts);
    const size_t smem = (size_t)nb * (LYA_NQ * sizeof(double) + sizeof(unsigned long long));
    const int64_t want = (n_pairs + 7) / 8;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, dev.sms));
    k_corr_noalloc<<<blocks, 256, smem, s>>>(p);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_noalloc_combine<<<(LYA_NQ * nb + 255) / 256, 256, 0, s>>>(nb, acc, hist);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return lya_fail(nullptr, LYA_ERR_CUDA, "lya_corr_pixel_noalloc: %s", cudaGetErrorString(e));
  return LYA_OK;
}
