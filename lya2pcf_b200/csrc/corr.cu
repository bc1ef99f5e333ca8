// Pair-binning kernels of the lya2pcf B200 library.
//
// Reference: pair_correlation (cuda_kernels.cpp:90-162), launched once per
// forest by two_point_per_pixel (correlation_procedures_pycuda.py:141-166).
// For every pixel pair (i in f1, j in f2) of a neighbouring forest pair:
//   cos12 = x1*x2 + y1*y2 + z1*z2, ch = sqrt(0.5(1+cos12)), sh = sqrt(0.5(1-cos12))
//   rp = |dc1-dc2| ch, rt = (dc1+dc2) sh, bp = floor(rp np/rpmax), bt = floor(rt nt/rtmax)
//   in range: W[bp,bt] += w1 w2, DW[bp,bt] += dw1 dw2
// plus the outputs the reference lacks: pair count, sum w1w2 rp, sum w1w2 rt,
// sum w1w2 (z1+z2)/2.
//
// B200 design:
// * One persistent launch over the whole work queue.  Each CTA owns a
//   contiguous, cost-balanced range of forest pairs; its warps pull pairs from
//   that range through a shared-memory counter.  Pairs are grouped by owner
//   slot, so the CTA accumulates one slot at a time in a shared-memory FP64
//   histogram and flushes it to global memory only when the slot changes,
//   through compensated (hi, lo) FP64 atomics.
// * A forest pair is walked along diagonals j - i = m (constant wavelength
//   offset on a common grid).  Along a diagonal |dc1-dc2| and dc1+dc2 change
//   slowly, so (bp, bt) stays constant for tens of steps: each lane keeps the
//   running sums of its current bin in registers and touches shared memory only
//   when the bin changes.  With sorted dc the walk is limited to the diagonal
//   band that can reach rp < rpmax, and a diagonal stops once rt >= rtmax.
// * FP32-guarded kernel: rp and rt are evaluated in FP32 from dc = hi + lo
//   (two floats) with cos/sin of the half angle computed once per forest pair
//   in FP64 exactly as the reference does.  A bin is accepted from FP32 only
//   when both coordinates are at least `guard` (bin units) away from a bin edge;
//   otherwise the pair is re-evaluated with the reference's FP64 formula.  The
//   guard is checked on the host against a proven bound on the FP32 error, so
//   every bin index (and hence every pair count) equals the FP64 formula's.
#include <cub/device/device_scan.cuh>
#include <thrust/binary_search.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/scan.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "lya_internal.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct CorrParams {
  const float4* __restrict__ pix4;
  const double4* __restrict__ pix8;
  const float* __restrict__ z32;
  const double* __restrict__ dc;
  const double* __restrict__ w;
  const double* __restrict__ dw;
  const double* __restrict__ z;
  const int64_t* __restrict__ pstart;
  const int32_t* __restrict__ len;
  const uint8_t* __restrict__ sorted;
  const int32_t* __restrict__ slot;
  const double* __restrict__ ux;
  const double* __restrict__ uy;
  const double* __restrict__ uz;
  const int32_t* __restrict__ f1;
  const int32_t* __restrict__ f2;
  const int64_t* __restrict__ cta_begin;
  double binner_rp, binner_rt;
  double inv_binner_rp, inv_binner_rt;
  int np, nt, nb;
  float gx, gy;        // guard half-widths in bin units (FP32 kernel)
  int cos_variant;
  int run_cap;
  int variant;          // walk: 0 default, 1 one diagonal per lane, 2 two diagonals per lane
  int inject_error;     // test hook: block 0 raises the device error flag (lya_debug_inject)
  double* hist;                 // [slot][LYA_NQ][2][nb]
  unsigned long long* counts;   // [slot][nb]
  unsigned long long* stats;    // [ST_N]
};

struct LaneStats {
  unsigned long long evaluated = 0, recheck = 0, runs = 0, inrange = 0;
};

// Shared-memory histogram of the slot being accumulated.
struct SmemHist {
  double* q;                  // [LYA_NQ][nb]
  unsigned int* n;            // [nb] pair counts (native 32-bit shared atomics)
  unsigned long long* gc;     // [nb] global counts of the slot being accumulated
  unsigned long long* err;    // device error flags (stats[ST_ERROR]): bit 0 = a record outside the histogram
};

// Count n more pairs in bin b: a 32-bit shared counter whose wrap-around is
// carried into the slot's global 64-bit count, so counts stay exact.
__device__ __forceinline__ void count_pairs(const SmemHist& h, int b, unsigned int n) {
  const unsigned int old = atomicAdd(&h.n[b], n);
  if (old > 0xffffffffu - n) atomicAdd(&h.gc[b], 1ull << 32);
}

__device__ __forceinline__ void pair_half_angles(const CorrParams& p, int a, int b, double& ch, double& sh) {
  double c = lya_cos12(p.ux[a], p.uy[a], p.uz[a], p.ux[b], p.uy[b], p.uz[b], p.cos_variant);
  // Rounding can push cos12 past 1 for coincident lines of sight; the
  // reference then takes sqrt of a negative number.  Clamp: rt = 0.
  c = fmin(1.0, fmax(-1.0, c));
  ch = __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(1.0, c)));
  sh = __dsqrt_rn(__dmul_rn(0.5, __dsub_rn(1.0, c)));
}

// Exact FP64 bin of a pixel pair (the reference formula); -1 when out of range.
__device__ __forceinline__ int bin_fp64(const CorrParams& p, double d1, double d2, double ch, double sh,
                                        double& rp, double& rt) {
  rp = __dmul_rn(fabs(__dsub_rn(d1, d2)), ch);
  rt = __dmul_rn(__dadd_rn(d1, d2), sh);
  const double fp = floor(__dmul_rn(rp, p.binner_rp));
  const double ft = floor(__dmul_rn(rt, p.binner_rt));
  if (fp >= 0.0 && fp < (double)p.np && ft >= 0.0 && ft < (double)p.nt) return (int)fp * p.nt + (int)ft;
  return -1;
}

// Diagonal band [m_lo, m_hi] of a forest pair with sorted dc: every pixel pair
// that can land in range has m = j - i inside it.  hi2(j) returns f2's dc_hi.
template <typename HiLoad>
__device__ void diagonal_band(int L1, int L2, const float4* __restrict__ P1, HiLoad hi2, double rp_reach,
                              double rt_reach, int& m_lo, int& m_hi) {
  const int lane = threadIdx.x & 31;
  int lo = INT_MAX, hi = INT_MIN;
  for (int i = lane; i < L1; i += 32) {
    const double d1 = (double)P1[i].x;
    const double margin = 1e-3 + 1e-6 * fabs(d1);
    const double tlo = d1 - rp_reach - margin;
    const double thi = fmin(d1 + rp_reach, rt_reach - d1) + margin;
    // first j with hi2[j] > tlo
    int a = 0, b = L2;
    while (a < b) { int mid = (a + b) >> 1; if ((double)hi2(mid) > tlo) b = mid; else a = mid + 1; }
    const int jlo = a;
    // last j with hi2[j] < thi
    a = jlo; b = L2;
    while (a < b) { int mid = (a + b) >> 1; if ((double)hi2(mid) < thi) a = mid + 1; else b = mid; }
    const int jhi = a - 1;
    if (jlo <= jhi) {
      lo = min(lo, jlo - i);
      hi = max(hi, jhi - i);
    }
  }
  lo = __reduce_min_sync(FULL, lo);
  hi = __reduce_max_sync(FULL, hi);
  m_lo = lo;
  m_hi = hi;
}

// ------------------------------------------------------------------ run records
// A lane's run (consecutive pairs of one diagonal in one bin) ends when the bin
// changes.  The lane appends the run's sums to its warp's record buffer in
// shared memory (plain stores, positions from a ballot); the warp drains the
// buffer into the CTA histogram with all 32 lanes when it holds 32 records or
// more, so the long-latency FP64 shared atomics never run in a divergent branch.
constexpr int REC = 128;   // records per warp buffer (up to 64 written per step)

struct __align__(16) RecF32 {
  int bin, n;
  float aw, adw, ax, ay, az, pad;
};
struct __align__(16) RecF64 {
  int bin, n;
  double aw, adw, ax, ay, az;
};

template <typename Rec>
__device__ __forceinline__ void drain(Rec* buf, int cnt, const SmemHist& h, int nb, LaneStats& st) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
  for (int k = lane; k < cnt; k += 32) {
    const Rec r = buf[k];
    if ((unsigned)r.bin >= (unsigned)nb || r.n <= 0) {   // never written by a correct walk: report, skip
      atomicOr(h.err, 1ull);
      continue;
    }
    st.runs++;
    st.inrange += (unsigned long long)r.n;
    atomicAdd(&h.q[0 * nb + r.bin], (double)r.aw);
    atomicAdd(&h.q[1 * nb + r.bin], (double)r.adw);
    atomicAdd(&h.q[2 * nb + r.bin], (double)r.ax);
    atomicAdd(&h.q[3 * nb + r.bin], (double)r.ay);
    atomicAdd(&h.q[4 * nb + r.bin], (double)r.az);
    count_pairs(h, r.bin, (unsigned int)r.n);
  }
  __syncwarp();
}

// ------------------------------------------------------------------ diagonal walk
// Lane layout: the 32 lanes of a warp walk 32 diagonals m = mg + 2*lane (two
// passes, mg even/odd offsets, cover a block of 64 diagonals) placed on one
// anti-diagonal: at step k lane l holds the pair (i, j) = (base+k-l, base+k+mg+l).
// Every lane then has the same i + j, hence nearly the same dc1 + dc2 and the
// same rt: rt-bin crossings and the rtmax stop happen for the whole warp at
// once.  rp-bin crossings (|dc1-dc2| drifts slowly along a diagonal) are
// handled by shifting the run's bin by +-1 in rp, without re-deriving it.
//
// Run state of a lane: bin (bx, by; bx < 0 = out of range), its acceptance
// interval [xlo, xhi) x [ylo, yhi) in bin units, the step k0 the run started
// and the running sums.  Traits supply the arithmetic precision.

struct TrF32 {
  using Real = float;
  using Rec = RecF32;
  struct Pix { float4 q; float z; };
  struct Geo { float chb, shb; };
  struct Ptr { const float4* __restrict__ q; const float* __restrict__ z; };
  static __device__ __forceinline__ Ptr ptr(const CorrParams& p, int64_t off) { return Ptr{p.pix4 + off, p.z32 + off}; }
  static __device__ __forceinline__ Pix load(const Ptr& a, int k) {
    Pix v;
    v.q = a.q[k];
    v.z = a.z[k];
    return v;
  }
  static __device__ __forceinline__ void coords(const Geo& g, const Pix& a, const Pix& b, float& x, float& y,
                                                float&, float&) {
    x = fabsf((a.q.x - b.q.x) + (a.q.y - b.q.y)) * g.chb;
    y = (a.q.x + b.q.x) * g.shb;
  }
  struct Acc {
    float aw, adw, ax, ay, az;
    __device__ __forceinline__ void zero() { aw = adw = ax = ay = az = 0.f; }
    __device__ __forceinline__ void add(const Pix& a, const Pix& b, float x, float y, float, float) {
      const float w12 = a.q.z * b.q.z;
      aw += w12;
      adw = fmaf(a.q.w, b.q.w, adw);
      ax = fmaf(w12, x, ax);
      ay = fmaf(w12, y, ay);
      az = fmaf(w12, a.z + b.z, az);
    }
  };
};

struct TrF64 {
  using Real = double;
  using Rec = RecF64;
  using Pix = double4;   // (dc, w, dw, z)
  struct Geo { double ch, sh, brp, brt; };
  using Ptr = const double4* __restrict__;
  static __device__ __forceinline__ Ptr ptr(const CorrParams& p, int64_t off) { return p.pix8 + off; }
  static __device__ __forceinline__ Pix load(Ptr a, int k) { return a[k]; }
  static __device__ __forceinline__ void coords(const Geo& g, const Pix& a, const Pix& b, double& x, double& y,
                                                double& rp, double& rt) {
    rp = __dmul_rn(fabs(__dsub_rn(a.x, b.x)), g.ch);
    rt = __dmul_rn(__dadd_rn(a.x, b.x), g.sh);
    x = __dmul_rn(rp, g.brp);
    y = __dmul_rn(rt, g.brt);
  }
  struct Acc {
    double aw, adw, ax, ay, az;
    __device__ __forceinline__ void zero() { aw = adw = ax = ay = az = 0.0; }
    __device__ __forceinline__ void add(const Pix& a, const Pix& b, double, double, double rp, double rt) {
      const double w12 = __dmul_rn(a.y, b.y);
      aw += w12;
      adw = __fma_rn(a.z, b.z, adw);
      ax = __fma_rn(w12, rp, ax);
      ay = __fma_rn(w12, rt, ay);
      az = __fma_rn(w12, __dadd_rn(a.w, b.w), az);
    }
  };
};

template <class Real>
struct Run {
  int bx, by, k0;
  Real xlo, xhi, ylo, yhi;
};

template <class Real>
__device__ __forceinline__ Real inf_of();
template <>
__device__ __forceinline__ float inf_of<float>() { return __int_as_float(0x7f800000); }
template <>
__device__ __forceinline__ double inf_of<double>() { return __longlong_as_double(0x7ff0000000000000ll); }

// Full classification of the pair starting a run.  FP32: accept the FP32 bin
// when both coordinates are at least the guard away from a bin edge (the edge
// at 0 cannot be crossed); otherwise take the bin from the reference FP64
// formula (d1p/d2p point at the pixels' FP64 data).  FP64: exact floor.
template <class Real>
__device__ __forceinline__ void classify(const CorrParams& p, Run<Real>& r, Real x, Real y, Real gx, Real gy,
                                         const double4* __restrict__ d1p, const double4* __restrict__ d2p,
                                         double ch, double sh, LaneStats& st) {
  const Real INF = inf_of<Real>();
  const Real npf = (Real)p.np, ntf = (Real)p.nt;
  if (!(x >= (Real)0) || !(y >= (Real)0)) {  // NaN or negative: excluded, re-examined every step
    r.bx = -1; r.by = -1; r.xlo = INF; r.xhi = -INF; r.ylo = INF; r.yhi = -INF;
    return;
  }
  if (y >= ntf + gy) {  // clearly beyond rtmax
    r.bx = -1; r.by = -1; r.xlo = -INF; r.xhi = INF; r.ylo = ntf + gy; r.yhi = INF;
    return;
  }
  if (x >= npf + gx) {  // clearly beyond rpmax
    r.bx = -1; r.by = -1; r.xlo = npf + gx; r.xhi = INF; r.ylo = -INF; r.yhi = INF;
    return;
  }
  const Real fx = floor(x), fy = floor(y);
  const bool safe = (fx == (Real)0 || x - fx >= gx) && (fx + (Real)1 - x > gx) &&
                    (fy == (Real)0 || y - fy >= gy) && (fy + (Real)1 - y > gy);
  if (safe) {
    r.xlo = fx == (Real)0 ? -INF : fx + gx; r.xhi = fx + (Real)1 - gx;
    r.ylo = fy == (Real)0 ? -INF : fy + gy; r.yhi = fy + (Real)1 - gy;
    if (fx < npf && fy < ntf) { r.bx = (int)fx; r.by = (int)fy; }
    else { r.bx = -1; r.by = -1; }
    return;
  }
  // FP32 only (gx = gy = 0 makes every FP64 pair safe): inside the guard band
  // the reference FP64 formula decides; the next pair is classified again.
  double rp, rt;
  const int k = bin_fp64(p, d1p->x, d2p->x, ch, sh, rp, rt);
  if (k >= 0) { r.bx = k / p.nt; r.by = k - r.bx * p.nt; } else { r.bx = -1; r.by = -1; }
  r.xlo = INF; r.xhi = -INF; r.ylo = INF; r.yhi = -INF;
  st.recheck++;
}

template <class Tr>
__device__ __forceinline__ void put_record(typename Tr::Rec* buf, int pos, int bin, int n, const typename Tr::Acc& a) {
  typename Tr::Rec rec;
  rec.bin = bin; rec.n = n; rec.aw = a.aw; rec.adw = a.adw; rec.ax = a.ax; rec.ay = a.ay; rec.az = a.az;
  buf[pos] = rec;
}

// Close the runs of the lanes in `who` at step k (records for in-range runs).
template <class Tr>
__device__ __forceinline__ void close_runs(bool who, Run<typename Tr::Real>& r, const typename Tr::Acc& acc, int k,
                                           int nt, typename Tr::Rec* buf, int& cnt, unsigned lt, LaneStats& st) {
  const bool wr = who && r.bx >= 0 && k > r.k0;
  const unsigned rb = __ballot_sync(FULL, wr);
  if (wr) put_record<Tr>(buf, cnt + __popc(rb & lt), r.bx * nt + r.by, k - r.k0, acc);
  cnt += __popc(rb);
}

template <class Tr, bool GUARDED>
__device__ void item_diag(const CorrParams& p, int64_t t, const SmemHist& h, typename Tr::Rec* buf, int& cnt,
                          LaneStats& st) {
  using Real = typename Tr::Real;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int fa = p.f1[t], fb = p.f2[t];
  const int L1 = p.len[fa], L2 = p.len[fb];
  if (L1 <= 0 || L2 <= 0) return;
  const int64_t a = p.pstart[fa], b = p.pstart[fb];
  const int np = p.np, nt = p.nt, nb = p.nb;
  double ch, sh;
  pair_half_angles(p, fa, fb, ch, sh);
  typename Tr::Geo geo;
  if constexpr (GUARDED) {
    geo.chb = __double2float_rn(ch * p.binner_rp);
    geo.shb = __double2float_rn(sh * p.binner_rt);
  } else {
    geo.ch = ch; geo.sh = sh; geo.brp = p.binner_rp; geo.brt = p.binner_rt;
  }
  const Real gx = GUARDED ? (Real)p.gx : (Real)0, gy = GUARDED ? (Real)p.gy : (Real)0;
  const bool srt = p.sorted[fa] && p.sorted[fb];
  int m_lo = -(L1 - 1), m_hi = L2 - 1;
  if (srt) {
    const float4* __restrict__ P1 = p.pix4 + a;
    const float4* __restrict__ P2 = p.pix4 + b;
    const double slack = GUARDED ? 2.0 * p.gx : 1e-3;
    const double rp_reach = ch > 0.0 ? ((double)np + slack) / (ch * p.binner_rp) : 1e300;
    const double rt_reach = sh > 0.0 ? ((double)nt + slack) / (sh * p.binner_rt) : 1e300;
    diagonal_band(L1, L2, P1, [&](int j) { return P2[j].x; }, rp_reach, rt_reach, m_lo, m_hi);
  }
  const Real INF = inf_of<Real>();
  const Real ycut = (Real)nt + gy;
  const int cap = p.run_cap;   // power of two
  for (int mb = m_lo; mb <= m_hi; mb += 64) {
    for (int par = 0; par < 2; ++par) {
      const int mg = mb + par;
      const int m = mg + 2 * lane;
      const int i_lo = max(0, -m);
      const int i_hi = (m <= m_hi) ? min(L1, L2 - m) : i_lo;
      const bool nonempty = i_lo < i_hi;
      int base = nonempty ? i_lo + lane : INT_MAX;
      base = __reduce_min_sync(FULL, base);
      if (base == INT_MAX) continue;
      const int k_beg = i_lo + lane - base;           // lane's first step
      int stop = nonempty ? i_hi + lane - base : 0;   // lane's end (exclusive), shrinks on the rtmax stop
      int k_end = stop;
      k_end = __reduce_max_sync(FULL, k_end);
      const int ioff = base - lane;            // i = ioff + k   (>= -31)
      const int joff = base + mg + lane;       // j = joff + k   (>= -31)
      // lane pointers at step 0; loads run up to 34 pixels outside a forest,
      // which stays inside the LYA_MARGIN-padded arrays
      const typename Tr::Ptr A1 = Tr::ptr(p, a + ioff);
      const typename Tr::Ptr A2 = Tr::ptr(p, b + joff);
      Run<Real> r;
      r.bx = -1; r.by = -1; r.k0 = 0; r.xlo = INF; r.xhi = -INF; r.ylo = INF; r.yhi = -INF;
      typename Tr::Acc acc;
      acc.zero();
      typename Tr::Pix q1 = Tr::load(A1, 0), q2 = Tr::load(A2, 0);
#pragma unroll 2
      for (int k = 0; k < k_end; ++k) {
        const typename Tr::Pix n1 = Tr::load(A1, k + 1), n2 = Tr::load(A2, k + 1);
        bool act = k >= k_beg && k < stop;
        Real x, y, rp, rt;
        Tr::coords(geo, q1, q2, x, y, rp, rt);
        const bool exl = x < r.xlo, exh = !(x < r.xhi), eyl = y < r.ylo, eyh = !(y < r.yhi);
        const bool slow = act && (exl || exh || eyl || eyh);
        if (__any_sync(FULL, slow)) {
          close_runs<Tr>(slow, r, acc, k, nt, buf, cnt, lt, st);
          if (slow) {
            acc.zero();
            r.k0 = k;
            bool full = true;
            // rp crossing into the adjacent bin, rt unchanged: shift the run by one in rp
            if (!eyl && !eyh && r.bx >= 0) {
              const int nbx = exh ? r.bx + 1 : r.bx - 1;
              // acceptance interval of bin nbx (the lower edge of bin 0 cannot be crossed)
              const Real nlo = nbx == 0 ? -INF : (Real)nbx + gx;
              const Real nhi = (Real)(nbx + 1) - gx;
              if (nbx >= 0 && nbx < np && x >= nlo && x < nhi) {
                r.bx = nbx; r.xlo = nlo; r.xhi = nhi;
                full = false;
              }
            }
            if (full) {
              if (srt && y >= ycut) {   // rt only grows along a sorted diagonal: lane done
                stop = k;
                act = false;
                r.bx = -1;
              } else {
                classify<Real>(p, r, x, y, gx, gy, p.pix8 + a + ioff + k, p.pix8 + b + joff + k, ch, sh, st);
              }
            }
          }
          if (cnt > REC - 32) {
            drain(buf, cnt, h, nb, st);
            cnt = 0;
          }
        }
        if (act) acc.add(q1, q2, x, y, rp, rt);
        q1 = n1;
        q2 = n2;
        if ((k & (cap - 1)) == cap - 1) {   // bound the length of a register sum
          const bool live = k >= k_beg && k < stop;
          close_runs<Tr>(live, r, acc, k + 1, nt, buf, cnt, lt, st);
          if (live) { acc.zero(); r.k0 = k + 1; }
          if (cnt > REC - 32) {
            drain(buf, cnt, h, nb, st);
            cnt = 0;
          }
          if (__all_sync(FULL, k + 1 >= stop)) break;
        }
      }
      st.evaluated += (unsigned long long)max(0, min(stop, k_end) - k_beg);
      const int kfin = min(stop, k_end);
      close_runs<Tr>(true, r, acc, max(kfin, r.k0), nt, buf, cnt, lt, st);
      if (cnt > REC - 32) {
        drain(buf, cnt, h, nb, st);
        cnt = 0;
      }
    }
  }
}

// Two diagonals per lane: lane l walks diagonals m = mg + 2l and m + 1 at the
// same f1 pixel i = base + k - l, so one pass covers 64 diagonals, the f1 pixel
// serves both pairs and the second pair's f2 pixel at step k is the first
// pair's at step k+1 (one f2 load per step).  Two independent runs per lane
// give the scheduler two dependency chains.  A bin change costs a predicated
// record store and, for an rp crossing into the adjacent bin, a predicated
// shift of the run; only rt crossings (warp-synchronous), guard-band pairs and
// range changes take the warp-voted full classification.
template <class Tr>
struct Walk2 {
  using Real = typename Tr::Real;
  using Pix = typename Tr::Pix;
  const CorrParams& p;
  const SmemHist& h;
  typename Tr::Rec* buf;
  int& cnt;
  LaneStats& st;
  typename Tr::Geo geo;
  Real gx, gy, ycut, INF;
  int np, nt, nb;
  unsigned lt;
  bool srt;
  const double4* __restrict__ D1;   // FP64 pixels of f1 at i = 0 (guard recheck)
  const double4* __restrict__ D2;   // FP64 pixels of f2 at j = 0
  double ch, sh;
  int ioff, joff;
  int ka_beg, kb_beg, stop_a, stop_b;
  Run<Real> ra, rb;
  typename Tr::Acc acca, accb;

  __device__ __forceinline__ void record(bool w, const Run<Real>& r, const typename Tr::Acc& acc, int k,
                                         unsigned bal, int base_pos) {
    if (w) {
      typename Tr::Rec rec;
      rec.bin = r.bx * nt + r.by; rec.n = k - r.k0;
      rec.aw = acc.aw; rec.adw = acc.adw; rec.ax = acc.ax; rec.ay = acc.ay; rec.az = acc.az;
      buf[base_pos + __popc(bal & lt)] = rec;
    }
  }

  // rp crossing into the adjacent bin with rt unchanged: returns true when the
  // run could be shifted (the pair lies inside the new bin's acceptance interval)
  __device__ __forceinline__ bool shift(Run<Real>& r, bool slow, bool eyl, bool eyh, bool exh, Real x) {
    const int nbx = exh ? r.bx + 1 : r.bx - 1;
    const Real nlo = nbx == 0 ? -INF : (Real)nbx + gx;
    const Real nhi = (Real)(nbx + 1) - gx;
    const bool ok = slow && !eyl && !eyh && r.bx >= 0 && (unsigned)nbx < (unsigned)np && x >= nlo && x < nhi;
    r.bx = ok ? nbx : r.bx;
    r.xlo = ok ? nlo : r.xlo;
    r.xhi = ok ? nhi : r.xhi;
    return ok;
  }

  __device__ __forceinline__ void full(Run<Real>& r, int& stop, bool& act, int k, Real x, Real y, int joff_pair) {
    if (srt && y >= ycut) {   // rt only grows along a sorted diagonal: the lane's diagonal is done
      stop = k;
      act = false;
      r.bx = -1;
    } else {
      classify<Real>(p, r, x, y, gx, gy, D1 + ioff + k, D2 + joff_pair + k, ch, sh, st);
    }
  }

  __device__ __forceinline__ void step(int k, const Pix& q1, const Pix& q2a, const Pix& q2b) {
    bool act_a = k >= ka_beg && k < stop_a;
    bool act_b = k >= kb_beg && k < stop_b;
    Real xa, ya, rpa, rta, xb, yb, rpb, rtb;
    Tr::coords(geo, q1, q2a, xa, ya, rpa, rta);
    Tr::coords(geo, q1, q2b, xb, yb, rpb, rtb);
    const bool exha = !(xa < ra.xhi), eyla = ya < ra.ylo, eyha = !(ya < ra.yhi);
    const bool exhb = !(xb < rb.xhi), eylb = yb < rb.ylo, eyhb = !(yb < rb.yhi);
    const bool slow_a = act_a && (xa < ra.xlo || exha || eyla || eyha);
    const bool slow_b = act_b && (xb < rb.xlo || exhb || eylb || eyhb);
    if (__any_sync(FULL, slow_a || slow_b)) {
      const bool wa = slow_a && ra.bx >= 0 && k > ra.k0;
      const bool wb = slow_b && rb.bx >= 0 && k > rb.k0;
      const unsigned bala = __ballot_sync(FULL, wa), balb = __ballot_sync(FULL, wb);
      record(wa, ra, acca, k, bala, cnt);
      record(wb, rb, accb, k, balb, cnt + __popc(bala));
      cnt += __popc(bala) + __popc(balb);
      const bool fa = slow_a && !shift(ra, slow_a, eyla, eyha, exha, xa);
      const bool fb = slow_b && !shift(rb, slow_b, eylb, eyhb, exhb, xb);
      if (slow_a) { acca.zero(); ra.k0 = k; }
      if (slow_b) { accb.zero(); rb.k0 = k; }
      if (__any_sync(FULL, fa || fb)) {
        if (fa) full(ra, stop_a, act_a, k, xa, ya, joff);
        if (fb) full(rb, stop_b, act_b, k, xb, yb, joff + 1);
      }
      if (cnt > REC - 64) {
        drain(buf, cnt, h, nb, st);
        cnt = 0;
      }
    }
    if (act_a) acca.add(q1, q2a, xa, ya, rpa, rta);
    if (act_b) accb.add(q1, q2b, xb, yb, rpb, rtb);
  }

  // close both runs at step k (all lanes in `live_*`), records for in-range ones
  __device__ __forceinline__ void close(bool live_a, bool live_b, int ka, int kb) {
    const bool wa = live_a && ra.bx >= 0 && ka > ra.k0;
    const bool wb = live_b && rb.bx >= 0 && kb > rb.k0;
    const unsigned bala = __ballot_sync(FULL, wa), balb = __ballot_sync(FULL, wb);
    record(wa, ra, acca, ka, bala, cnt);
    record(wb, rb, accb, kb, balb, cnt + __popc(bala));
    cnt += __popc(bala) + __popc(balb);
    if (live_a) { acca.zero(); ra.k0 = ka; }
    if (live_b) { accb.zero(); rb.k0 = kb; }
    if (cnt > REC - 64) {
      drain(buf, cnt, h, nb, st);
      cnt = 0;
    }
  }
};

template <class Tr, bool GUARDED>
__device__ void item_diag2(const CorrParams& p, int64_t t, const SmemHist& h, typename Tr::Rec* buf, int& cnt,
                           LaneStats& st) {
  using Real = typename Tr::Real;
  using Pix = typename Tr::Pix;
  const int lane = threadIdx.x & 31;
  const int fa = p.f1[t], fb = p.f2[t];
  const int L1 = p.len[fa], L2 = p.len[fb];
  if (L1 <= 0 || L2 <= 0) return;
  const int64_t a = p.pstart[fa], b = p.pstart[fb];
  Walk2<Tr> W{p, h, buf, cnt, st};
  W.np = p.np; W.nt = p.nt; W.nb = p.nb;
  W.lt = (1u << lane) - 1u;
  pair_half_angles(p, fa, fb, W.ch, W.sh);
  if constexpr (GUARDED) {
    W.geo.chb = __double2float_rn(W.ch * p.binner_rp);
    W.geo.shb = __double2float_rn(W.sh * p.binner_rt);
  } else {
    W.geo.ch = W.ch; W.geo.sh = W.sh; W.geo.brp = p.binner_rp; W.geo.brt = p.binner_rt;
  }
  W.gx = GUARDED ? (Real)p.gx : (Real)0;
  W.gy = GUARDED ? (Real)p.gy : (Real)0;
  W.INF = inf_of<Real>();
  W.ycut = (Real)W.nt + W.gy;
  W.srt = p.sorted[fa] && p.sorted[fb];
  W.D1 = p.pix8 + a;
  W.D2 = p.pix8 + b;
  int m_lo = -(L1 - 1), m_hi = L2 - 1;
  if (W.srt) {
    const float4* __restrict__ P1 = p.pix4 + a;
    const float4* __restrict__ P2 = p.pix4 + b;
    const double slack = GUARDED ? 2.0 * p.gx : 1e-3;
    const double rp_reach = W.ch > 0.0 ? ((double)W.np + slack) / (W.ch * p.binner_rp) : 1e300;
    const double rt_reach = W.sh > 0.0 ? ((double)W.nt + slack) / (W.sh * p.binner_rt) : 1e300;
    diagonal_band(L1, L2, P1, [&](int j) { return P2[j].x; }, rp_reach, rt_reach, m_lo, m_hi);
  }
  const int cap = p.run_cap;   // power of two, even
  for (int mg = m_lo; mg <= m_hi; mg += 64) {
    const int ma = mg + 2 * lane, mb = ma + 1;
    // pair a: (i, i + ma), pair b: (i, i + mb); i = base + k - lane
    const int ia_lo = max(0, -ma), ia_hi = (ma <= m_hi) ? min(L1, L2 - ma) : ia_lo;
    const int ib_lo = max(0, -mb), ib_hi = (mb <= m_hi) ? min(L1, L2 - mb) : ib_lo;
    const bool ne_a = ia_lo < ia_hi, ne_b = ib_lo < ib_hi;
    int base = min(ne_a ? ia_lo + lane : INT_MAX, ne_b ? ib_lo + lane : INT_MAX);
    base = __reduce_min_sync(FULL, base);
    if (base == INT_MAX) continue;
    W.ka_beg = ne_a ? ia_lo + lane - base : 0;
    W.kb_beg = ne_b ? ib_lo + lane - base : 0;
    W.stop_a = ne_a ? ia_hi + lane - base : 0;
    W.stop_b = ne_b ? ib_hi + lane - base : 0;
    int k_end = max(W.stop_a, W.stop_b);
    k_end = __reduce_max_sync(FULL, k_end);
    W.ioff = base - lane;             // i = ioff + k    (>= -31)
    W.joff = base + ma - lane;        // j_a = joff + k  (>= -31), j_b = j_a + 1
    const typename Tr::Ptr A1 = Tr::ptr(p, a + W.ioff);
    const typename Tr::Ptr A2 = Tr::ptr(p, b + W.joff);
    W.ra.bx = -1; W.ra.by = -1; W.ra.k0 = 0;
    W.ra.xlo = W.INF; W.ra.xhi = -W.INF; W.ra.ylo = W.INF; W.ra.yhi = -W.INF;
    W.rb = W.ra;
    W.acca.zero();
    W.accb.zero();
    // pixels of steps k (q1a, q2x, q2y); the loop body handles two steps so the
    // registers rotate without copies
    Pix q1a = Tr::load(A1, 0), q2x = Tr::load(A2, 0), q2y = Tr::load(A2, 1);
    int k = 0;
    for (; k < k_end; k += 2) {
      const Pix q1b = Tr::load(A1, k + 1), q2z = Tr::load(A2, k + 2);
      W.step(k, q1a, q2x, q2y);
      q1a = Tr::load(A1, k + 2);
      q2x = Tr::load(A2, k + 3);
      if (k + 1 < k_end) W.step(k + 1, q1b, q2y, q2z);
      // now q1a = f1[k+2], q2x = f2[k+3]; the next pair of steps wants (f2[k+2], f2[k+3])
      q2y = q2x;
      q2x = q2z;
      if (((k + 2) & (cap - 1)) == 0) {   // bound the length of a register sum
        W.close(k + 1 >= W.ka_beg && k + 1 < W.stop_a, k + 1 >= W.kb_beg && k + 1 < W.stop_b, k + 2, k + 2);
        if (__all_sync(FULL, k + 2 >= W.stop_a && k + 2 >= W.stop_b)) { k += 2; break; }
      }
    }
    const int kfa = min(W.stop_a, k_end), kfb = min(W.stop_b, k_end);
    st.evaluated += (unsigned long long)(max(0, kfa - W.ka_beg) + max(0, kfb - W.kb_beg));
    W.close(true, true, max(kfa, W.ra.k0), max(kfb, W.rb.k0));
  }
}

// ------------------------------------------------------------------ lean walk (FP32, both forests lean)
// Same lane layout as item_diag2 (lane l: diagonals m = mg + 2l and m + 1 at
// f1 pixel i = base + k - l), for forest pairs whose dc are sorted, finite and
// in [0, LYA_LEAN_DC_MAX).  The bin tests run on the FP32 pixel coordinates
// themselves:
//   e = |(hi1 - hi2) + (lo1 - lo2)|  ~ |dc1 - dc2|,    s = hi1 + hi2  ~ dc1 + dc2
// against per-forest-pair FP32 threshold tables built with directed rounding:
//   e >= tlo[b]  =>  X64 >= b,   e < thi[b]  =>  X64 < b + 1,   e >= tout => X64 >= np
// (X64 the reference's FP64 bin coordinate of rp; likewise slo, shi, scut for
// rt and s), tlo[b] = RU((b + g)/cx), thi[b] = RD((b + 1 - g)/cx), cx = ch*np/rpmax,
// g the guard in bin units.  |e - |dc1-dc2|| <= 2^-23 |dc1-dc2| + 2^-45 (dc1+dc2)
// and |s - (dc1+dc2)| <= 2^-23 (dc1+dc2) (|lo| <= 2^-24 hi), so every
// accepted bin is the FP64 formula's bin when g is at least
// (n+1)(2^-23 + 2^-50)*1.1 + 1e-7 bins (2.7e-5 Mpc/h for 50 bins of 4 Mpc/h),
// below the bound the host already enforces for the other walks.
// s is non-decreasing along a diagonal of two sorted forests, so the rt test is
// one-sided and a diagonal ends for good once s >= scut.  A run's state is its
// bin and its interval [tlo, thi) x [.., shi); a pair outside the interval is
// an event: the run is closed (record), shifted to the adjacent rp or rt bin
// when the pair lies inside that bin's interval, otherwise classified again
// (tables, or the reference FP64 formula inside the guard band).  Sums run over
// e and s and are scaled to bin units (x = e*cx, y = s*cy) when a run is
// recorded.  Each lane's first run is classified before the walk, so ragged
// diagonal starts cost no event; each step takes one warp vote for events (two
// pairs per lane), and the loop body holds two steps so the pixel registers
// rotate without copies.
// Per-warp state of the forest pair being walked, in shared memory (read on
// the rare paths only, so the walk's registers hold just the runs, the sums and
// the pixels); the threshold tables follow it: tlo[np], thi[np], slo[nt], shi[nt].
struct __align__(16) LeanCtl {
  double ch, sh;
  const double4* d1;     // FP64 pixels of f1 (i = 0)
  const double4* d2;     // FP64 pixels of f2 (j = 0)
  float tout, scut;      // e >= tout: beyond rpmax;  s >= scut: beyond rtmax
  float cxf, cyf;        // FP32 copies of cx, cy: candidate bins and record scaling
  int base, mg;          // current pass: f1 pixel i = base + k - lane, f2 pixel j = base + mg + lane + k
  int pad0, pad1;
};
constexpr int LEAN_CTL_FLOATS = (int)(sizeof(LeanCtl) / sizeof(float));
// floats per warp: the state and the tables, rounded to keep the next warp's state 16-byte aligned
__host__ __device__ __forceinline__ int lean_ctl_stride(int np, int nt) {
  return LEAN_CTL_FLOATS + ((2 * (np + nt) + 3) & ~3);
}

__device__ __forceinline__ float* lean_tab(LeanCtl* c) { return reinterpret_cast<float*>(c + 1); }

struct LeanRun {
  int bx, by, k0;
  float tlo, thi, shi;
};

struct LeanAcc {
  float aw, adw, ae, as, az;
  __device__ __forceinline__ void zero() { aw = adw = ae = as = az = 0.f; }
  __device__ __forceinline__ void add(const float4& a, float za, const float4& b, float zb, float e, float s) {
    const float w12 = a.z * b.z;
    aw += w12;
    adw = fmaf(a.w, b.w, adw);
    ae = fmaf(w12, e, ae);
    as = fmaf(w12, s, as);
    az = fmaf(w12, za + zb, az);
  }
};

__device__ __forceinline__ float lean_e(const float4& a, const float4& b) { return fabsf((a.x - b.x) + (a.y - b.y)); }
__device__ __forceinline__ float lean_s(const float4& a, const float4& b) { return a.x + b.x; }

// true when the pair (e, s) lies outside the run's interval (NaN-safe form)
__device__ __forceinline__ bool lean_out(const LeanRun& r, float e, float s) {
  return !(e >= r.tlo) || !(e < r.thi) || !(s < r.shi);
}

// Per-forest-pair state and threshold tables of one warp.
__device__ __forceinline__ void lean_setup(LeanCtl* c, double ch, double sh, const double4* d1, const double4* d2,
                                           const CorrParams& p) {
  const int lane = threadIdx.x & 31;
  __syncwarp();   // every lane is done with the previous forest pair's state
  const double cx = __dmul_rn(ch, p.binner_rp), cy = __dmul_rn(sh, p.binner_rt);
  const double gx = (double)p.gx, gy = (double)p.gy;
  float* tlo = lean_tab(c);
  float* thi = tlo + p.np;
  float* slo = thi + p.np;
  float* shi = slo + p.nt;
  for (int b = lane; b < p.np; b += 32) {
    tlo[b] = b == 0 ? -1.0f : __double2float_ru(__ddiv_ru((double)b + gx, cx));
    thi[b] = __double2float_rd(__ddiv_rd((double)(b + 1) - gx, cx));
  }
  for (int b = lane; b < p.nt; b += 32) {
    slo[b] = b == 0 ? -1.0f : __double2float_ru(__ddiv_ru((double)b + gy, cy));
    shi[b] = __double2float_rd(__ddiv_rd((double)(b + 1) - gy, cy));
  }
  if (lane == 0) {
    c->ch = ch; c->sh = sh; c->d1 = d1; c->d2 = d2;
    c->tout = __double2float_ru(__ddiv_ru((double)p.np + gx, cx));
    c->scut = __double2float_ru(__ddiv_ru((double)p.nt + gy, cy));
    c->cxf = __double2float_rn(cx);
    c->cyf = __double2float_rn(cy);
  }
  __syncwarp();
}

// Full classification of the pair (e, s) at step k of diagonal dm (0: a, 1: b)
// of this lane, which starts a run.  Sets the lane's diagonal end kend = k when
// the diagonal is past rtmax.
__device__ __forceinline__ void lean_classify(const CorrParams& p, const LeanCtl* c, LeanRun& r, float e, float s,
                                           int& kend, int k, int dm, LaneStats& st) {
  const float INF = __int_as_float(0x7f800000);
  const float* tlo = lean_tab(const_cast<LeanCtl*>(c));
  const float* thi = tlo + p.np;
  const float* slo = thi + p.np;
  const float* shi = slo + p.nt;
  const float scut = c->scut, tout = c->tout;
  if (!(s < scut)) {   // past rtmax for good (s only grows): the diagonal is done
    kend = k;
    r.bx = -1; r.by = -1; r.tlo = -INF; r.thi = INF; r.shi = INF;
    return;
  }
  if (e >= tout) {     // beyond rpmax; |dc1-dc2| may shrink again
    r.bx = -1; r.by = -1; r.tlo = tout; r.thi = INF; r.shi = scut;
    return;
  }
  const int cbx = min((int)(e * c->cxf), p.np - 1);
  const int cby = min((int)(s * c->cyf), p.nt - 1);
  const float tl = tlo[cbx], th = thi[cbx], sl = slo[cby], su = shi[cby];
  if (e >= tl && e < th && s >= sl && s < su) {
    r.bx = cbx; r.by = cby; r.tlo = tl; r.thi = th; r.shi = su;
    return;
  }
  // guard band (or an FP32 candidate one bin off): the reference FP64 formula
  // decides this pair; the empty interval re-examines the next one
  const int lane = threadIdx.x & 31;
  const int i = c->base - lane + k, j = c->base + c->mg + lane + k + dm;
  double rp, rt;
  const int b = bin_fp64(p, c->d1[i].x, c->d2[j].x, c->ch, c->sh, rp, rt);
  if (b >= 0) { r.bx = b / p.nt; r.by = b - r.bx * p.nt; } else { r.bx = -1; r.by = -1; }
  r.tlo = INF; r.thi = -INF; r.shi = -INF;
  st.recheck++;
}

// Move the run to the adjacent bin the pair (e, s) lies in, when one rp or one
// rt edge was crossed; false when a full classification is needed.
__device__ __forceinline__ bool lean_shift(const CorrParams& p, const LeanCtl* c, LeanRun& r, float e, float s) {
  const float INF = __int_as_float(0x7f800000);
  if (r.bx < 0) return false;
  const bool xo = !(e >= r.tlo) || !(e < r.thi);
  const bool yo = !(s < r.shi);
  if (xo == yo) return false;
  const float* tlo = lean_tab(const_cast<LeanCtl*>(c));
  if (xo) {
    const int nbx = e >= r.thi ? r.bx + 1 : r.bx - 1;
    if (nbx >= p.np) {
      const float tout = c->tout;
      if (!(e >= tout)) return false;
      r.bx = -1; r.by = -1; r.tlo = tout; r.thi = INF; r.shi = c->scut;
      return true;
    }
    if (nbx < 0) return false;
    const float tl = tlo[nbx], th = tlo[p.np + nbx];
    if (!(e >= tl && e < th)) return false;
    r.bx = nbx; r.tlo = tl; r.thi = th;
    return true;
  }
  const int nby = r.by + 1;
  if (nby >= p.nt) return false;
  const float sl = tlo[2 * p.np + nby], su = tlo[2 * p.np + p.nt + nby];
  if (!(s >= sl && s < su)) return false;
  r.by = nby; r.shi = su;
  return true;
}

struct LeanWalk {
  const CorrParams& p;
  LeanCtl* c;
  const SmemHist& h;
  RecF32* buf;
  int& cnt;
  LaneStats& st;
  int ka_beg, kb_beg, ka_end, kb_end;
  int kall;   // last step any lane of the warp still walks (exclusive)
  LeanRun ra, rb;
  LeanAcc acca, accb;

  __device__ __forceinline__ void record(bool w, const LeanRun& r, const LeanAcc& acc, int k, unsigned bal, int pos) {
    if (w) {
      const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
      RecF32 rec;
      rec.bin = r.bx * p.nt + r.by; rec.n = k - r.k0;
      rec.aw = acc.aw; rec.adw = acc.adw; rec.ax = acc.ae * c->cxf; rec.ay = acc.as * c->cyf; rec.az = acc.az;
      rec.pad = 0.f;
      buf[pos + __popc(bal & lt)] = rec;
    }
  }

  // close both runs at step ka / kb for the lanes in live_*; records for in-range runs
  __device__ __forceinline__ void close(bool live_a, bool live_b, int ka, int kb) {
    const bool wa = live_a && ra.bx >= 0 && ka > ra.k0;
    const bool wb = live_b && rb.bx >= 0 && kb > rb.k0;
    const unsigned bala = __ballot_sync(FULL, wa), balb = __ballot_sync(FULL, wb);
    record(wa, ra, acca, ka, bala, cnt);
    record(wb, rb, accb, kb, balb, cnt + __popc(bala));
    cnt += __popc(bala) + __popc(balb);
    if (live_a) { acca.zero(); ra.k0 = ka; }
    if (live_b) { accb.zero(); rb.k0 = kb; }
    if (cnt > REC - 64) {
      drain(buf, cnt, h, p.nb, st);
      cnt = 0;
    }
  }

  // One step: pair a = (q1, qa), pair b = (q1, qb), with the warp's events.
  // There is no event-free fast path: with 64 diagonals per warp and runs of
  // about 30 pairs, some lane leaves its run on almost every step, so a
  // warp-wide "no event" test before the step costs more than it saves.
  __device__ __forceinline__ void step(int k, const float4& q1, float z1, const float4& qa, float za,
                                            const float4& qb, float zb) {
    const float ea = lean_e(q1, qa), sa = lean_s(q1, qa);
    const float eb = lean_e(q1, qb), sb = lean_s(q1, qb);
    bool act_a = k >= ka_beg && k < ka_end;
    bool act_b = k >= kb_beg && k < kb_end;
    const bool exa = act_a && lean_out(ra, ea, sa);
    const bool exb = act_b && lean_out(rb, eb, sb);
    if (__any_sync(FULL, exa || exb)) {
      const bool wa = exa && ra.bx >= 0 && k > ra.k0;
      const bool wb = exb && rb.bx >= 0 && k > rb.k0;
      const unsigned bala = __ballot_sync(FULL, wa), balb = __ballot_sync(FULL, wb);
      record(wa, ra, acca, k, bala, cnt);
      record(wb, rb, accb, k, balb, cnt + __popc(bala));
      cnt += __popc(bala) + __popc(balb);
      const bool fa = exa && !lean_shift(p, c, ra, ea, sa);
      const bool fb = exb && !lean_shift(p, c, rb, eb, sb);
      if (exa) { acca.zero(); ra.k0 = k; }
      if (exb) { accb.zero(); rb.k0 = k; }
      if (__any_sync(FULL, fa || fb)) {
        if (fa) lean_classify(p, c, ra, ea, sa, ka_end, k, 0, st);
        if (fb) lean_classify(p, c, rb, eb, sb, kb_end, k, 1, st);
        act_a = act_a && k < ka_end;
        act_b = act_b && k < kb_end;
        int ke = max(ka_end, kb_end);   // diagonals past rtmax shorten the walk
        ke = __reduce_max_sync(FULL, ke);
        kall = min(kall, ke);
      }
      if (cnt > REC - 64) {
        drain(buf, cnt, h, p.nb, st);
        cnt = 0;
      }
    }
    if (act_a) acca.add(q1, z1, qa, za, ea, sa);
    if (act_b) accb.add(q1, z1, qb, zb, eb, sb);
  }
};

__device__ void item_lean(const CorrParams& p, int64_t t, const SmemHist& h, RecF32* buf, LeanCtl* ctl, int& cnt,
                          LaneStats& st) {
  const int lane = threadIdx.x & 31;
  const int fa = p.f1[t], fb = p.f2[t];
  const int L1 = p.len[fa], L2 = p.len[fb];
  if (L1 <= 0 || L2 <= 0) return;
  const int64_t a = p.pstart[fa], b = p.pstart[fb];
  int m_lo, m_hi;
  {
    double ch, sh;
    pair_half_angles(p, fa, fb, ch, sh);
    lean_setup(ctl, ch, sh, p.pix8 + a, p.pix8 + b, p);
    const float4* __restrict__ P1 = p.pix4 + a;
    const float4* __restrict__ P2 = p.pix4 + b;
    const double slack = 2.0 * p.gx;
    const double rp_reach = ch > 0.0 ? ((double)p.np + slack) / (ch * p.binner_rp) : 1e300;
    const double rt_reach = sh > 0.0 ? ((double)p.nt + slack) / (sh * p.binner_rt) : 1e300;
    diagonal_band(L1, L2, P1, [&](int j) { return P2[j].x; }, rp_reach, rt_reach, m_lo, m_hi);
  }
  LeanWalk W{p, ctl, h, buf, cnt, st};
  const int cap = p.run_cap;   // power of two, even
  for (int mg = m_lo; mg <= m_hi; mg += 64) {
    const int ma = mg + 2 * lane, mb = ma + 1;
    const int ia_lo = max(0, -ma), ia_hi = (ma <= m_hi) ? min(L1, L2 - ma) : ia_lo;
    const int ib_lo = max(0, -mb), ib_hi = (mb <= m_hi) ? min(L1, L2 - mb) : ib_lo;
    const bool ne_a = ia_lo < ia_hi, ne_b = ib_lo < ib_hi;
    int base = min(ne_a ? ia_lo + lane : INT_MAX, ne_b ? ib_lo + lane : INT_MAX);
    base = __reduce_min_sync(FULL, base);
    if (base == INT_MAX) continue;
    W.ka_beg = ne_a ? ia_lo + lane - base : 0;
    W.kb_beg = ne_b ? ib_lo + lane - base : 0;
    W.ka_end = ne_a ? ia_hi + lane - base : 0;
    W.kb_end = ne_b ? ib_hi + lane - base : 0;
    int k_end = max(W.ka_end, W.kb_end);
    k_end = __reduce_max_sync(FULL, k_end);
    W.kall = k_end;
    __syncwarp();
    if (lane == 0) { ctl->base = base; ctl->mg = mg; }
    __syncwarp();
    const int ioff = base - lane;        // i = ioff + k    (>= -31)
    const int joff = base + mg + lane;   // j_a = joff + k  (>= -31), j_b = j_a + 1
    const float4* __restrict__ A1 = p.pix4 + a + ioff;
    const float* __restrict__ Z1 = p.z32 + a + ioff;
    const float4* __restrict__ A2 = p.pix4 + b + joff;
    const float* __restrict__ Z2 = p.z32 + b + joff;
    // each lane's first run, classified before the walk
    W.acca.zero();
    W.accb.zero();
    {
      const float INF = __int_as_float(0x7f800000);
      W.ra.bx = -1; W.ra.by = -1; W.ra.tlo = INF; W.ra.thi = -INF; W.ra.shi = -INF;
      W.rb = W.ra;
      W.ra.k0 = W.ka_beg;
      W.rb.k0 = W.kb_beg;
      if (ne_a) {
        const int k = W.ka_beg;
        const float4 u = A1[k], v = A2[k];
        lean_classify(p, ctl, W.ra, lean_e(u, v), lean_s(u, v), W.ka_end, k, 0, st);
      }
      if (ne_b) {
        const int k = W.kb_beg;
        const float4 u = A1[k], v = A2[k + 1];
        lean_classify(p, ctl, W.rb, lean_e(u, v), lean_s(u, v), W.kb_end, k, 1, st);
      }
      int ke = max(W.ka_end, W.kb_end);   // first runs past rtmax
      ke = __reduce_max_sync(FULL, ke);
      W.kall = min(W.kall, ke);
    }
    // steps k, k+1 per iteration: f1 pixels q1a (k), q1b (k+1); f2 pixels
    // q2x (k), q2y (k+1), q2z (k+2).  Pairs: a@k = (q1a, q2x), b@k = (q1a, q2y),
    // a@k+1 = (q1b, q2y), b@k+1 = (q1b, q2z).
    float4 q1a = A1[0], q2x = A2[0], q2y = A2[1];
    float z1a = Z1[0], z2x = Z2[0], z2y = Z2[1];
    int k = 0;
    for (; k < W.kall; k += 2) {
      const float4 q1b = A1[k + 1], q2z = A2[k + 2];
      const float z1b = Z1[k + 1], z2z = Z2[k + 2];
      W.step(k, q1a, z1a, q2x, z2x, q2y, z2y);
      W.step(k + 1, q1b, z1b, q2y, z2y, q2z, z2z);
      q1a = A1[k + 2];
      z1a = Z1[k + 2];
      q2x = q2z;
      z2x = z2z;
      q2y = A2[k + 3];
      z2y = Z2[k + 3];
      // registers now hold f1[k+2], f2[k+2], f2[k+3]: the next iteration's pixels
      if (((k + 2) & (cap - 1)) == 0) {   // bound the length of a register sum
        W.close(k + 1 >= W.ka_beg && k + 1 < W.ka_end, k + 1 >= W.kb_beg && k + 1 < W.kb_end, k + 2, k + 2);
        if (__all_sync(FULL, k + 2 >= W.ka_end && k + 2 >= W.kb_end)) { k += 2; break; }
      }
    }
    const int kfa = min(W.ka_end, k_end), kfb = min(W.kb_end, k_end);
    st.evaluated += (unsigned long long)(max(0, kfa - W.ka_beg) + max(0, kfb - W.kb_beg));
    W.close(true, true, max(kfa, W.ra.k0), max(kfb, W.rb.k0));
  }
}

// ------------------------------------------------------------------ FP64 plain (every pixel pair)
__device__ void item_plain(const CorrParams& p, int64_t t, const SmemHist& h, LaneStats& st) {
  const int lane = threadIdx.x & 31;
  const int fa = p.f1[t], fb = p.f2[t];
  const int L1 = p.len[fa], L2 = p.len[fb];
  if (L1 <= 0 || L2 <= 0) return;
  const int64_t a = p.pstart[fa], b = p.pstart[fb];
  double ch, sh;
  pair_half_angles(p, fa, fb, ch, sh);
  for (int i = 0; i < L1; ++i) {
    const double4 q1 = p.pix8[a + i];
    for (int j = lane; j < L2; j += 32) {
      const double4 q2 = p.pix8[b + j];
      double rp, rt;
      const int k = bin_fp64(p, q1.x, q2.x, ch, sh, rp, rt);
      st.evaluated++;
      if (k >= 0) {
        const double w12 = __dmul_rn(q1.y, q2.y);
        atomicAdd(&h.q[0 * p.nb + k], w12);
        atomicAdd(&h.q[1 * p.nb + k], __dmul_rn(q1.z, q2.z));
        atomicAdd(&h.q[2 * p.nb + k], __dmul_rn(w12, rp));
        atomicAdd(&h.q[3 * p.nb + k], __dmul_rn(w12, rt));
        atomicAdd(&h.q[4 * p.nb + k], __dmul_rn(w12, __dadd_rn(q1.w, q2.w)));
        count_pairs(h, k, 1u);
        st.inrange++;
      }
    }
  }
}

// ------------------------------------------------------------------ persistent driver
// Compensated accumulation of v into the (hi, lo) pair at hi/lo: the atomic
// returns the old hi, the rounding error of hi + v is recovered exactly
// (TwoSum) and added to lo.
__device__ __forceinline__ void add_compensated(double* hi, double* lo, double v) {
  const double old = atomicAdd(hi, v);
  const double s = old + v;
  const double bb = s - old;
  const double err = (old - (s - bb)) + (v - bb);
  if (err != 0.0) atomicAdd(lo, err);
}

template <int KIND>
constexpr size_t rec_bytes() {
  return KIND == LYA_KERNEL_FP32_GUARDED ? sizeof(RecF32) : (KIND == LYA_KERNEL_FP64_DIAGONAL ? sizeof(RecF64) : 0);
}

// Walk selection of a pair-kernel instance.  The FP32 kernel runs as one
// instance with the lean walk only (pairs of two lean forests; the others are
// skipped) followed, when the catalogue has forests the lean walk cannot take,
// by one with the two-diagonal walk for exactly those pairs, so each instance
// carries one walk's code; WALK_ANY takes every pair with the walk
// p.variant names.
enum { WALK_ANY = 0, WALK_LEAN = 1, WALK_REST = 2 };

template <int KIND, int WARPS, int WALK>
__global__ void __launch_bounds__(WARPS * 32, 1) k_corr(const CorrParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nb = p.nb;
  SmemHist h;
  h.q = reinterpret_cast<double*>(smem);
  h.n = reinterpret_cast<unsigned int*>(h.q + LYA_NQ * nb);
  h.gc = nullptr;
  h.err = p.stats + ST_ERROR;
  if (p.inject_error && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(h.err, 2ull);
  // the count array keeps 8 bytes per bin so the record buffers stay 16-byte aligned
  unsigned char* bufs = reinterpret_cast<unsigned char*>(h.q + LYA_NQ * nb) + (size_t)nb * sizeof(unsigned long long);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* mybuf = bufs + (size_t)warp * REC * rec_bytes<KIND>();
  // lean walk: per-warp state and threshold tables after the record buffers
  LeanCtl* myctl = reinterpret_cast<LeanCtl*>(reinterpret_cast<float*>(bufs + (size_t)WARPS * REC * rec_bytes<KIND>()) +
                                              (size_t)warp * lean_ctl_stride(p.np, p.nt));
  __shared__ unsigned long long s_next;
  __shared__ long long s_seg_end;
  __shared__ int s_slot;

  for (int k = threadIdx.x; k < LYA_NQ * nb; k += blockDim.x) h.q[k] = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) h.n[k] = 0u;
  LaneStats st;
  int cnt = 0;   // records pending in this warp's buffer (warp-uniform)
  const int64_t begin = p.cta_begin[blockIdx.x], end = p.cta_begin[blockIdx.x + 1];
  int64_t seg = begin;
  __syncthreads();
  while (seg < end) {
    if (threadIdx.x == 0) {
      const int s = p.slot[p.f1[seg]];
      int64_t lo = seg + 1, hi = end;   // first item of a later slot
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (p.slot[p.f1[mid]] > s) hi = mid; else lo = mid + 1;
      }
      s_seg_end = lo;
      s_slot = s;
      s_next = (unsigned long long)seg;
    }
    __syncthreads();
    const int64_t seg_end = s_seg_end;
    const int slot = s_slot;
    h.gc = p.counts + (size_t)slot * nb;
    for (;;) {
      unsigned long long t = 0;
      if (lane == 0) t = atomicAdd(&s_next, 1ull);
      t = __shfl_sync(FULL, t, 0);
      if ((int64_t)t >= seg_end) break;
      if (KIND == LYA_KERNEL_FP32_GUARDED) {
        if (WALK == WALK_LEAN) {
          if (p.sorted[p.f1[t]] & p.sorted[p.f2[t]] & LYA_LEAN)
            item_lean(p, (int64_t)t, h, reinterpret_cast<RecF32*>(mybuf), myctl, cnt, st);
        } else if (WALK == WALK_REST) {
          if (!(p.sorted[p.f1[t]] & p.sorted[p.f2[t]] & LYA_LEAN))
            item_diag2<TrF32, true>(p, (int64_t)t, h, reinterpret_cast<RecF32*>(mybuf), cnt, st);
        } else if (p.variant == 1) {
          item_diag<TrF32, true>(p, (int64_t)t, h, reinterpret_cast<RecF32*>(mybuf), cnt, st);
        } else {
          item_diag2<TrF32, true>(p, (int64_t)t, h, reinterpret_cast<RecF32*>(mybuf), cnt, st);
        }
      } else if (KIND == LYA_KERNEL_FP64_DIAGONAL) {
        if (p.variant == 2) item_diag2<TrF64, false>(p, (int64_t)t, h, reinterpret_cast<RecF64*>(mybuf), cnt, st);
        else item_diag<TrF64, false>(p, (int64_t)t, h, reinterpret_cast<RecF64*>(mybuf), cnt, st);
      }
      else item_plain(p, (int64_t)t, h, st);
    }
    if (KIND == LYA_KERNEL_FP32_GUARDED) drain(reinterpret_cast<RecF32*>(mybuf), cnt, h, nb, st);
    if (KIND == LYA_KERNEL_FP64_DIAGONAL) drain(reinterpret_cast<RecF64*>(mybuf), cnt, h, nb, st);
    cnt = 0;
    __syncthreads();
    double* gh = p.hist + (size_t)slot * LYA_NQ * 2 * nb;
    for (int k = threadIdx.x; k < LYA_NQ * nb; k += blockDim.x) {
      const int q = k / nb, bb = k - q * nb;
      double v = h.q[k];
      if (v != 0.0) {
        // the FP32 kernel sums w12*x in bin units; all kernels sum w12*(z1+z2)
        if (KIND == LYA_KERNEL_FP32_GUARDED && q == 2) v *= p.inv_binner_rp;
        if (KIND == LYA_KERNEL_FP32_GUARDED && q == 3) v *= p.inv_binner_rt;
        if (q == 4) v *= 0.5;
        add_compensated(gh + (size_t)(q * 2) * nb + bb, gh + (size_t)(q * 2 + 1) * nb + bb, v);
      }
      h.q[k] = 0.0;
    }
    unsigned long long* gc = p.counts + (size_t)slot * nb;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      if (h.n[k]) atomicAdd(&gc[k], (unsigned long long)h.n[k]);
      h.n[k] = 0u;
    }
    __syncthreads();
    seg = seg_end;
  }
  // statistics: one atomic per warp
  unsigned long long e = st.evaluated, r = st.recheck, u = st.runs, n = st.inrange;
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(FULL, e, o);
    r += __shfl_xor_sync(FULL, r, o);
    u += __shfl_xor_sync(FULL, u, o);
    n += __shfl_xor_sync(FULL, n, o);
  }
  if (lane == 0) {
    atomicAdd(&p.stats[ST_EVALUATED], e);
    atomicAdd(&p.stats[ST_RECHECK], r);
    atomicAdd(&p.stats[ST_RUNS], u);
    atomicAdd(&p.stats[ST_INRANGE], n);
  }
}

template <int KIND, int WARPS>
size_t corr_smem_bytes(const CorrParams& p, int nb) {
  return (size_t)nb * (LYA_NQ * sizeof(double) + sizeof(unsigned long long)) +
         (size_t)WARPS * REC * rec_bytes<KIND>() +
         (KIND == LYA_KERNEL_FP32_GUARDED ? (size_t)WARPS * lean_ctl_stride(p.np, p.nt) * sizeof(float) : 0);
}

template <int KIND, int WARPS, int WALK>
cudaError_t set_corr_smem(const CorrParams& p, int nb) {
  return cudaFuncSetAttribute(k_corr<KIND, WARPS, WALK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)corr_smem_bytes<KIND, WARPS>(p, nb));
}

template <int KIND, int WARPS, int WALK>
cudaError_t launch_corr(const CorrParams& p, int nctas, int nb, cudaStream_t s) {
  k_corr<KIND, WARPS, WALK><<<nctas, WARPS * 32, corr_smem_bytes<KIND, WARPS>(p, nb), s>>>(p);
  return cudaGetLastError();
}

// The FP32 kernel's default walk: the lean instance, plus the two-diagonal
// instance for the pairs it skips when the catalogue has forests it cannot take.
static bool fp32_lean_walk(int variant) { return variant == 0 || variant == 3; }

// ------------------------------------------------------------------ CTA ranges
__global__ void k_item_cost(int64_t n, const int32_t* __restrict__ f1, const int32_t* __restrict__ f2,
                            const int32_t* __restrict__ len, long long* __restrict__ cost) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    cost[k] = (long long)len[f1[k]] * (long long)len[f2[k]];
}

// first item k in [lo, hi) whose first forest's slot is >= s (items are grouped
// by first forest, slots non-decreasing in forest order)
__device__ int64_t first_item_of_slot(const int32_t* __restrict__ f1, const int32_t* __restrict__ slot, int64_t lo,
                                      int64_t hi, int s) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (slot[f1[mid]] < s) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// CTA b takes items [out[b], out[b+1]): equal shares of the reference pair
// count inside the item range of slots [slot_begin, slot_end).
__global__ void k_cta_bounds(int nctas, int64_t n, const long long* __restrict__ prefix,
                             const int32_t* __restrict__ f1, const int32_t* __restrict__ slot, int slot_begin,
                             int slot_end, int64_t* __restrict__ out, double* __restrict__ range_pairs) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > nctas) return;
  const bool all = slot_begin == 0 && slot_end == 0;
  const int64_t it_lo = all ? 0 : first_item_of_slot(f1, slot, 0, n, slot_begin);
  const int64_t it_hi = all ? n : first_item_of_slot(f1, slot, it_lo, n, slot_end);
  const long long base = it_lo > 0 ? prefix[it_lo - 1] : 0;
  const long long total = it_hi > it_lo ? prefix[it_hi - 1] - base : 0;
  if (b == 0) { out[0] = it_lo; *range_pairs = (double)total; return; }
  if (b == nctas) { out[b] = it_hi; return; }
  const long long target = base + (long long)((double)total * ((double)b / nctas));
  int64_t lo = it_lo, hi = it_hi;   // first k with prefix[k] > target
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (prefix[mid] > target) hi = mid; else lo = mid + 1;
  }
  out[b] = lo;
}

}  // namespace

// Largest FP32 error of a bin coordinate (bin units) for coordinates below
// `reach` bins: four roundings of relative size 2^-24 (hi-difference and lo sum,
// the FP32 factor ch*binner, the product) bound |x - x64| by 2^-22 x; the
// FP64 reference value itself carries < 2^-51 x.  Margin 10%, plus the
// rounding of the interval ends fx + guard in FP32 (half an ulp of reach).
static double guard_bound_bins(double reach) {
  const double rel = std::ldexp(1.0, -22) + std::ldexp(1.0, -50);
  const double ulp_reach = std::ldexp(1.0, (int)std::floor(std::log2(std::max(reach, 1.0))) - 23);
  return 1.1 * rel * reach + ulp_reach + 1e-12;
}

// Everything a captured run depends on: the kernel parameters and the
// scratch and output buffers.  A run whose key differs from the captured one
// is captured again.
struct RunGraphKey {
  CorrParams p;
  int kind, nctas, nslots, nb;
  int slot_begin, slot_end;
  int rest_pass;          // FP32 lean walk: second instance for the pairs it skips
  int64_t n_items;
  const void* cost;
  const void* scan_tmp;
  size_t scan_bytes;
};

// The stream work of one run: clear the outputs, balance the work queue over
// the CTAs (cost prefix sum), the persistent pair kernel, and the copy of the
// counters to pinned host memory.  No allocation and no synchronisation, so it
// is captured once in a CUDA graph and replayed.
static cudaError_t enqueue_run(lya_ctx* ctx, const RunGraphKey& k, double* d_range_pairs, int slot_begin,
                               int slot_end) {
  cudaStream_t s = ctx->stream;
  const CorrParams& p = k.p;
  cudaError_t e = cudaEventRecordWithFlags(ctx->ev2, s, cudaEventRecordExternal);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(p.hist, 0, sizeof(double) * (size_t)k.nslots * LYA_NQ * 2 * k.nb, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(p.counts, 0, sizeof(unsigned long long) * (size_t)k.nslots * k.nb, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(p.stats, 0, sizeof(unsigned long long) * ST_N, s);
  if (e == cudaSuccess && k.n_items > 0) {
    const int blocks = (int)std::min<int64_t>((k.n_items + 255) / 256, (int64_t)ctx->num_sms * 16);
    k_item_cost<<<blocks, 256, 0, s>>>(k.n_items, p.f1, p.f2, p.len, ctx->cost);
    e = cudaGetLastError();
    size_t bytes = k.scan_bytes;
    if (e == cudaSuccess)
      e = cub::DeviceScan::InclusiveSum(ctx->scan_tmp, bytes, ctx->cost, ctx->cost, k.n_items, s);
  }
  if (e == cudaSuccess) {
    k_cta_bounds<<<(k.nctas + 1 + 127) / 128, 128, 0, s>>>(k.nctas, k.n_items, ctx->cost, p.f1, p.slot, slot_begin,
                                                             slot_end, ctx->cta_begin, d_range_pairs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev0, s, cudaEventRecordExternal);
  if (e == cudaSuccess) {
    if (k.kind == LYA_KERNEL_FP32_GUARDED && fp32_lean_walk(p.variant)) {
      e = launch_corr<LYA_KERNEL_FP32_GUARDED, 16, WALK_LEAN>(p, k.nctas, k.nb, s);
      if (e == cudaSuccess && k.rest_pass) e = launch_corr<LYA_KERNEL_FP32_GUARDED, 16, WALK_REST>(p, k.nctas, k.nb, s);
    } else if (k.kind == LYA_KERNEL_FP32_GUARDED) {
      e = launch_corr<LYA_KERNEL_FP32_GUARDED, 16, WALK_ANY>(p, k.nctas, k.nb, s);
    } else if (k.kind == LYA_KERNEL_FP64_DIAGONAL) {
      e = launch_corr<LYA_KERNEL_FP64_DIAGONAL, 16, WALK_ANY>(p, k.nctas, k.nb, s);
    } else {
      e = launch_corr<LYA_KERNEL_FP64_PLAIN, 16, WALK_ANY>(p, k.nctas, k.nb, s);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev1, s, cudaEventRecordExternal);
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev3, s, cudaEventRecordExternal);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->h_stats, p.stats, sizeof(unsigned long long) * ST_N, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->h_stats + ST_N, d_range_pairs, sizeof(double), cudaMemcpyDeviceToHost, s);
  return e;
}

int lya_corr_launch(lya_ctx* ctx, const lya_corr_opts* o) {
  const int kind = o->kernel;
  const int nb = ctx->np * ctx->nt;
  const int nslots = ctx->cat.n_slots;
  cudaStream_t s = ctx->stream;

  // guard check (FP32 kernel)
  const double gx_bins = o->guard * ctx->np / ctx->rpmax;
  const double gy_bins = o->guard * ctx->nt / ctx->rtmax;
  const double bx = guard_bound_bins(ctx->np + 1.0), by = guard_bound_bins(ctx->nt + 1.0);
  ctx->last.guard_bound = std::max(bx * ctx->rpmax / ctx->np, by * ctx->rtmax / ctx->nt);
  if (kind == LYA_KERNEL_FP32_GUARDED && (!(gx_bins >= bx) || !(gy_bins >= by) || gx_bins > 0.25 || gy_bins > 0.25))
    return lya_fail(ctx, LYA_ERR_GUARD,
                    "guard %.3g Mpc/h outside [%.3g, %.3g]: below the proven FP32 error bound or above a quarter bin",
                    o->guard, ctx->last.guard_bound, 0.25 * std::min(ctx->rpmax / ctx->np, ctx->rtmax / ctx->nt));

  // outputs and scratch (allocated once, reused by later runs)
  if (ctx->hist_slots != nslots || ctx->hist_nb != nb || !ctx->hist) {
    lya_free(ctx->hist); lya_free(ctx->counts);
    cudaError_t e = lya_alloc(&ctx->hist, (size_t)nslots * LYA_NQ * 2 * nb);
    if (e == cudaSuccess) e = lya_alloc(&ctx->counts, (size_t)nslots * nb);
    if (e != cudaSuccess) {
      lya_free(ctx->hist); lya_free(ctx->counts);
      ctx->hist_slots = 0;
      return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_run: output allocation failed");
    }
    ctx->hist_slots = nslots; ctx->hist_nb = nb;
  }
  const int nctas = ctx->num_sms * std::max(1, o->blocks_per_sm);
  if (ctx->cta_cap < nctas + 2) {
    lya_free(ctx->cta_begin);
    if (lya_alloc(&ctx->cta_begin, (size_t)nctas + 2) != cudaSuccess)
      return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_run: allocation failed");
    ctx->cta_cap = nctas + 2;
  }
  // the range's reference pair count shares the cta_begin buffer
  double* d_range_pairs = reinterpret_cast<double*>(ctx->cta_begin + nctas + 1);
  const int64_t n = ctx->wq.n_pairs;
  if (ctx->cost_cap < std::max<int64_t>(n, 1)) {
    lya_free(ctx->cost);
    ctx->cost_cap = 0;
    if (lya_alloc(&ctx->cost, (size_t)std::max<int64_t>(n, 1)) != cudaSuccess)
      return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_run: allocation of the cost buffer failed");
    ctx->cost_cap = std::max<int64_t>(n, 1);
  }
  size_t scan_bytes = 0;
  if (n > 0) {
    LYA_CHECK_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, ctx->cost, ctx->cost, n, s));
    if (scan_bytes > ctx->scan_tmp_bytes) {
      if (ctx->scan_tmp) cudaFree(ctx->scan_tmp);
      ctx->scan_tmp = nullptr;
      ctx->scan_tmp_bytes = 0;
      if (cudaMalloc(&ctx->scan_tmp, scan_bytes) != cudaSuccess)
        return lya_fail(ctx, LYA_ERR_ALLOC, "lya_corr_run: allocation of the scan scratch failed");
      ctx->scan_tmp_bytes = scan_bytes;
    }
  }

  RunGraphKey key;
  memset(&key, 0, sizeof(key));   // padding bytes take part in the comparison
  CorrParams& p = key.p;
  const DevCatalog& c = ctx->cat;
  p.pix4 = c.pix4; p.z32 = c.z32; p.pix8 = c.pix8; p.dc = c.dc; p.w = c.w; p.dw = c.dw; p.z = c.z;
  p.pstart = c.pstart; p.len = c.len; p.sorted = c.sorted; p.slot = c.slot;
  p.ux = c.ux; p.uy = c.uy; p.uz = c.uz;
  p.f1 = ctx->wq.f1; p.f2 = ctx->wq.f2; p.cta_begin = ctx->cta_begin;
  p.binner_rp = (double)ctx->np / ctx->rpmax;
  p.binner_rt = (double)ctx->nt / ctx->rtmax;
  p.inv_binner_rp = ctx->rpmax / (double)ctx->np;
  p.inv_binner_rt = ctx->rtmax / (double)ctx->nt;
  p.np = ctx->np; p.nt = ctx->nt; p.nb = nb;
  p.gx = (float)gx_bins; p.gy = (float)gy_bins;
  p.cos_variant = ctx->cos_variant;
  p.run_cap = o->run_cap > 0 ? o->run_cap : 128;
  p.variant = o->variant;
  p.inject_error = ctx->inject_device_error ? 1 : 0;
  ctx->inject_device_error = false;   // one run
  p.hist = ctx->hist; p.counts = ctx->counts; p.stats = ctx->stats;
  key.kind = kind; key.nctas = nctas; key.nslots = nslots; key.nb = nb; key.n_items = n;
  key.slot_begin = o->slot_begin; key.slot_end = o->slot_end;
  key.rest_pass = (kind == LYA_KERNEL_FP32_GUARDED && fp32_lean_walk(o->variant) && ctx->cat.n_not_lean > 0) ? 1 : 0;
  key.cost = ctx->cost; key.scan_tmp = ctx->scan_tmp; key.scan_bytes = scan_bytes;

  // shared-memory limit of the pair kernel: set outside any capture
  {
    cudaError_t e = cudaSuccess;
    if (kind == LYA_KERNEL_FP32_GUARDED) {
      e = set_corr_smem<LYA_KERNEL_FP32_GUARDED, 16, WALK_LEAN>(p, nb);
      if (e == cudaSuccess) e = set_corr_smem<LYA_KERNEL_FP32_GUARDED, 16, WALK_REST>(p, nb);
      if (e == cudaSuccess) e = set_corr_smem<LYA_KERNEL_FP32_GUARDED, 16, WALK_ANY>(p, nb);
    } else if (kind == LYA_KERNEL_FP64_DIAGONAL) {
      e = set_corr_smem<LYA_KERNEL_FP64_DIAGONAL, 16, WALK_ANY>(p, nb);
    } else {
      e = set_corr_smem<LYA_KERNEL_FP64_PLAIN, 16, WALK_ANY>(p, nb);
    }
    if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_corr_run: %s", cudaGetErrorString(e));
  }
  static_assert(sizeof(RunGraphKey) <= sizeof(ctx->run_graph_key), "graph key does not fit the context");
  if (!ctx->run_graph || memcmp(&ctx->run_graph_key, &key, sizeof(key)) != 0) {
    if (ctx->run_graph) { cudaGraphExecDestroy(ctx->run_graph); ctx->run_graph = nullptr; }
    cudaGraph_t g = nullptr;
    LYA_CHECK_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const cudaError_t eq = enqueue_run(ctx, key, d_range_pairs, key.slot_begin, key.slot_end);
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (eq != cudaSuccess || ec != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return lya_fail(ctx, LYA_ERR_CUDA, "lya_corr_run: capture failed: %s",
                      cudaGetErrorString(eq != cudaSuccess ? eq : ec));
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_corr_run: instantiate: %s", cudaGetErrorString(ei));
    ctx->run_graph = ex;
    memcpy(&ctx->run_graph_key, &key, sizeof(key));
  } else {
    ctx->graph_launches++;
  }
  LYA_CHECK_CUDA(ctx, cudaGraphLaunch(ctx->run_graph, s));
  // k_item_cost (when there are items), k_cta_bounds, the pair kernel (two instances with the rest pass)
  ctx->launches += (n > 0 ? 3 : 2) + key.rest_pass;
  LYA_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  float ms = 0.f, ms_all = 0.f;
  LYA_CHECK_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  LYA_CHECK_CUDA(ctx, cudaEventElapsedTime(&ms_all, ctx->ev2, ctx->ev3));
  const unsigned long long* hst = ctx->h_stats;
  double range_pairs = 0.0;
  memcpy(&range_pairs, hst + ST_N, sizeof(double));
  ctx->last.kernel_ms = ms;
  ctx->last.run_ms = ms_all;
  ctx->last.run_ref_pairs = range_pairs;
  ctx->last.evaluated_pairs = (double)hst[ST_EVALUATED];
  ctx->last.guard_rechecks = (double)hst[ST_RECHECK];
  ctx->last.runs_flushed = (double)hst[ST_RUNS];
  ctx->last.in_range_pairs = (double)hst[ST_INRANGE];
  if (hst[ST_ERROR]) {
    ctx->have_result = false;
    return lya_fail(ctx, LYA_ERR_DEVICE, "lya_corr_run: the pair kernel raised its error flag 0x%llx (%s)",
                    (unsigned long long)hst[ST_ERROR],
                    (hst[ST_ERROR] & 1) ? "a run record outside the histogram was dropped" : "injected by lya_debug_inject");
  }
  ctx->have_result = true;
  return LYA_OK;
}

extern "C" int lya_corr_run(lya_ctx* ctx, const lya_corr_opts* opts) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_corr_run: ctx is NULL");
  lya_corr_opts o{};
  o.kernel = LYA_KERNEL_FP32_GUARDED;
  o.guard = 1e-4;
  if (opts) o = *opts;
  if (o.kernel < 0 || o.kernel > 2) return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: unknown kernel %d", o.kernel);
  if (o.blocks_per_sm < 0 || o.blocks_per_sm > 1) return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: blocks_per_sm must be 0 or 1");
  if (o.variant < 0 || o.variant > 3) return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: variant must be 0, 1, 2 or 3");
  if (o.variant == 3 && o.kernel != LYA_KERNEL_FP32_GUARDED)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: variant 3 (lean walk) exists for the FP32 kernel only");
  if (o.kernel == LYA_KERNEL_FP32_GUARDED && (size_t)2 * (ctx->np + ctx->nt) > 1024)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: FP32 kernel needs np + nt <= 512 (threshold tables)");
  if (o.run_cap != 0 && (o.run_cap < 8 || o.run_cap > 1024 || (o.run_cap & (o.run_cap - 1)) != 0))
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: run_cap must be 0 or a power of two in [8, 1024]");
  if (o.warps_per_block != 0 && o.warps_per_block != 16)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: warps_per_block must be 0 or 16");
  if (o.slot_begin < 0 || o.slot_end < o.slot_begin || o.slot_end > ctx->cat.n_slots)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_corr_run: slot range [%d,%d) outside [0,%d]", o.slot_begin, o.slot_end,
                    ctx->cat.n_slots);
  if (!ctx->bins_set) return lya_fail(ctx, LYA_ERR_STATE, "lya_corr_run: call lya_set_bins first");
  if (ctx->cat.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_corr_run: no forests uploaded");
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  return lya_corr_launch(ctx, &o);
}
