// Distortion-matrix numerator of the lya2pcf B200 library.
//
// Reference: distortion_per_pixel (distortion_procedures_pycuda.py:195-279)
// with the kernels precompute_distances, compute_etas, order_active and
// compute_d (cuda_kernels.cpp:46-87, 165-278).  For a forest pair (f1, f2)
// and pixel pairs (i, j) in bin A, (k, l) in bin B, with
//   eta1_ik = delta_ik - w_k/Om1 - dl_i w_k dl_k / O1,   O = sum w dl^2,
// the reference scatters, per in-range pair and per active bin B,
//   D_AB += w_i w_j sum_{(k,l) in B} eta1_ik eta2_jl.
//
// This kernel evaluates the same sum in factored form.  With per-pixel columns
//   S2[A,i] = sum_{j:(i,j) in A} w_j,   L2[A,i] = sum_{j:(i,j) in A} w_j dl_j
//   S1[A,j] = sum_{i:(i,j) in A} w_i,   L1[A,j] = sum_{i:(i,j) in A} w_i dl_i
// and per-bin moments M0_A = sum w_i w_j, Mi_A = sum w_i dl_i w_j,
// Mj_A = sum w_i w_j dl_j, Mij_A = sum w_i dl_i w_j dl_j (over (i,j) in A):
//   D_AB = [A==B] M0_A
//        + M0_A M0_B/(Om1 Om2) + Mj_A Mj_B/(Om1 O2) + Mi_A Mi_B/(O1 Om2) + Mij_A Mij_B/(O1 O2)
//        - sum_i w_i (S2[A,i] S2[B,i]/Om2 + L2[A,i] L2[B,i]/O2)
//        - sum_j w_j (S1[A,j] S1[B,j]/Om1 + L1[A,j] L1[B,j]/O1)
// (expand eta1_ik eta2_jl; the delta terms give the diagonal, the products of
// the two projections the rank-4 part, the cross terms the columns).  The
// column of a pixel spans a few rt bins only, so the column products are
// 50x50 dense blocks (rp x rp) per pair of rt bins.
//
// One CTA per forest pair (dynamic queue).  Bins come from the reference FP64
// formula.  Phase 1: the columns of every pixel (a warp per pixel, lanes over
// its partners) go to CTA-private global scratch as dense [TS rt bins][np]
// rows.  Phase 2: the 50x50 (rp x rp) blocks (t, u) of D over the pair's window
// of rt bins, diagonal blocks first (they complete the moments of bin t, read
// from the same staged rows: the f1 weights placed in padding columns
// NS..NS+3 of the staged rows make accumulator rows NS..NS+3 of the diagonal
// block's MMAs the four moments, when NS + 4 <= 64; otherwise a loop over the
// staged rows).  A block whose rt bins are both spanned by some
// pixel column gets the column products as a small dense FP64 GEMM on the
// tensor cores: the rows of the pixels covering t and u are staged in shared
// memory in chunks of CH pixels, and each warp accumulates 16 x 8 tiles of the
// block (four tiles of 16 rp bins down, 8 across; mma.sync m16n8k8 f64, FP64
// having no tcgen05 kind; rows at or beyond np enter as zeros); the
// rank-4 and diagonal terms are added to the accumulators, and each D entry of
// the window gets one atomic add per forest pair (both (A, B) and (B, A): D is
// symmetric).
// A forest whose sum w dl^2 is 0 has no slope to project out: its slope terms
// are 0.
#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "lya_internal.cuh"

namespace {

constexpr int TS = 8;         // rt bins a pixel column may span
constexpr int TSB = TS + 2;   // rows of a column being built (its window may be one bin wider at each end)
constexpr int NP_MAX = 64;    // np of the blocks: at most 4 x 8 tiles of 16 x 8
// Launch shapes the autotuner chooses from: threads per CTA (DT) and pixels per
// staged chunk of a block (CH, a multiple of 8: the K of one MMA).  Shape 0 is the default.
struct DistShape { int dt, ch; };
constexpr DistShape DIST_SHAPES[] = {{512, 32}, {512, 16}, {512, 24}, {256, 32}, {256, 16}};
constexpr int N_DIST_SHAPES = sizeof(DIST_SHAPES) / sizeof(DIST_SHAPES[0]);
// Staged row length for np bins: 8 * ceil(np/8) plus 4, so the four rows of an
// MMA fragment load fall in disjoint shared-memory banks.
__host__ __device__ __forceinline__ int stage_npad(int np) { return 8 * ((np + 7) / 8) + 4; }
// Row stride of the column scratch: np rounded up to even, so every row starts
// on a 16-byte boundary (the asynchronous 16-byte copies of the staging).
__host__ __device__ __forceinline__ int col_stride(int np) { return (np + 1) & ~1; }
// Shared-memory doubles of the staging area: two buffers of four [CH][NPAD]
// row sets (double buffering), or the per-warp column builders of phase 1.
__host__ __device__ __forceinline__ int stage_doubles(int CH, int NW, int np) {
  const int a = 2 * 4 * CH * stage_npad(np), b = NW * 2 * (TS + 2) * np;
  return a > b ? a : b;
}

struct DistParams {
  const double4* __restrict__ pix8;   // (dc, w, dw, z)
  const double* __restrict__ dl;
  const int64_t* __restrict__ pstart;
  const int32_t* __restrict__ len;
  const uint8_t* __restrict__ sorted;
  const double* __restrict__ ux;
  const double* __restrict__ uy;
  const double* __restrict__ uz;
  const double* __restrict__ omega;
  const double* __restrict__ odl2;
  const int32_t* __restrict__ f1;
  const int32_t* __restrict__ f2;
  const long long* n_items;   // [1] forest pairs of the queue (device: the captured graph serves any count)
  int max_len;
  double binner_rp, binner_rt;
  int np, nt, nb, cos_variant;
  int npad;                // staged row length (stage_npad(np))
  double* col;             // scratch [grid][2 sides][max_len][TS][col_stride(np)] x {S, L}
  double* moments;         // scratch [grid][4][nt][np]: moments of the window's bins
  double* D;               // [nb][nb]
  double* W;               // [nb]
  unsigned long long* err; // [1] pixels whose column spans more than TS rt bins
  unsigned long long* next;// [1] work queue counter
  unsigned long long* mma; // [1] block-product work in m8n8k4 units (8x8 tiles, rows rounded to 4), for the roofline
  int shape;               // launch shape (DIST_SHAPES index); part of the captured graph's key
  int row_offsets;         // 1: the pixel list carries each pixel's scratch row offset (shared memory allows it)
};

// Bin of a pixel pair with the reference FP64 formula, as (bp, bt); false when
// out of range.
__device__ __forceinline__ bool pair_bin2(double d1, double d2, double ch, double sh, const DistParams& p, int& bp,
                                          int& bt) {
  const double rp = __dmul_rn(fabs(__dsub_rn(d1, d2)), ch);
  const double rt = __dmul_rn(__dadd_rn(d1, d2), sh);
  const double fp = floor(__dmul_rn(rp, p.binner_rp));
  const double ft = floor(__dmul_rn(rt, p.binner_rt));
  if (!(fp >= 0.0 && fp < (double)p.np && ft >= 0.0 && ft < (double)p.nt)) return false;
  bp = (int)fp;
  bt = (int)ft;
  return true;
}

// rt bin coordinate floor(rt * nt / rtmax) of a pixel pair (reference formula, unclamped)
__device__ __forceinline__ double pair_ft(double d1, double d2, double sh, const DistParams& p) {
  return floor(__dmul_rn(__dmul_rn(__dadd_rn(d1, d2), sh), p.binner_rt));
}

// First index in [lo, hi) of the sorted shared array a at which the monotone
// predicate holds (hi when it holds nowhere), found by the whole warp: 32
// probes and one vote per level, ceil(log32(hi - lo)) + 1 levels instead of
// log2(hi - lo) dependent steps of a binary search.
template <class Pred>
__device__ __forceinline__ int warp_first(const double* a, int lo, int hi, Pred pred) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const int step = (hi - lo + 31) >> 5;
    const int idx = lo + (lane + 1) * step - 1;
    const bool t = lane == 31 || idx >= hi || pred(a[idx]);   // the last lane closes the range
    const unsigned bal = __ballot_sync(0xffffffffu, t);
    const int f = __ffs(bal) - 1;
    const int pf = lo + (f + 1) * step - 1;     // lane f's probe (true, or the closing lane)
    const int nhi = (f == 31 || pf >= hi) ? hi : pf;
    lo += f * step;                             // lane f-1's probe was false
    hi = nhi;
  }
  const int idx = lo + lane;
  const unsigned bal = __ballot_sync(0xffffffffu, idx < hi && pred(a[idx]));
  return bal ? lo + __ffs(bal) - 1 : hi;
}

template <int DT, int CH>
__global__ void __launch_bounds__(DT, 1) k_dist(const DistParams p) {
  constexpr int NW = DT / 32;   // warps per CTA
  // 16 x 8 accumulator tiles per warp: NW/4 warps share each of the four tile
  // rows of 16 rp bins (np <= 64), and split its (at most 8) tile columns
  constexpr int CC = NW >= 16 ? 2 : 4;
  extern __shared__ __align__(16) unsigned char smem[];
  const int ML = p.max_len;
  const int np = p.np, nt = p.nt, nb = p.nb, NPAD = p.npad;
  double* sd = reinterpret_cast<double*>(smem);          // [2][ML] dc
  double* sw = sd + 2 * ML;                              // [2][ML] w
  double* sl = sw + 2 * ML;                              // [2][ML] dl
  double* ksc = sl + 2 * ML;                             // [2][ML] column-product weights k_S of a pixel
  double* klc = ksc + 2 * ML;                            // [2][ML] and k_L
  double* mom = p.moments + (size_t)blockIdx.x * 4 * nt * np;   // [4][nt][np] (CTA-private, L2-resident)
  double* stage = klc + 2 * ML;                          // 2 x [4][CH][NPAD] staged rows, or the column builders
  const int stage_len = stage_doubles(CH, NW, np);
  double* kbuf = stage + stage_len;                      // [2][4][CH] per staged row: k_S, k_L, f1 w, f1 w dl
  int* tlo = reinterpret_cast<int*>(kbuf + 8 * CH);      // [2][ML]
  int* span = tlo + 2 * ML;                              // [2][ML]
  int* plist = span + 2 * ML;                            // [2*ML] packed (side << 16 | pixel)
  int* roff = plist + 2 * ML;                            // [2*ML] scratch offset of a listed pixel's row t (row_offsets)
  __shared__ int s_T0, s_T1, s_maxspan, s_cnt;
  __shared__ long long s_item;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NS = col_stride(np);
  // q / (NS/2) as a multiply-high: exact for q < 2^16 (the copies of a chunk)
  const unsigned seg_magic = (unsigned)((0x100000000ull + (unsigned)(NS / 2) - 1) / (unsigned)(NS / 2));
  double* colS = p.col + (size_t)blockIdx.x * 2 * 2 * ML * TS * NS;   // [2 sides][ML][TS][NS]
  double* colL = colS + (size_t)2 * ML * TS * NS;
  double* myS = stage + (size_t)warp * 2 * TSB * np;
  double* myL = myS + TSB * np;
  const int ntile = (np + 7) / 8;   // tile rows = tile columns of a 50x50 block (7 for np = 50)
  // warp w: tile row mt = w mod 4 (rp bins 16 mt .. 16 mt + 15) and tile
  // columns ng, ng + nwm, ... (ng = w / 4) of 8 rp bins each
  const int nwm = NW / 4;
  const int mt = warp & 3, ng = warp >> 2;
  const int grp = lane >> 2, kq = lane & 3;
  unsigned long long n_mma = 0;     // thread 0: MMAs of this CTA

  for (;;) {
    if (tid == 0) s_item = (long long)atomicAdd(p.next, 1ull);
    __syncthreads();
    const long long t_item = s_item;
    if (t_item >= *p.n_items) break;
    const int a = p.f1[t_item], b = p.f2[t_item];
    const int L1 = p.len[a], L2 = p.len[b];
    if (L1 <= 0 || L2 <= 0) { __syncthreads(); continue; }
    double c = lya_cos12(p.ux[a], p.uy[a], p.uz[a], p.ux[b], p.uy[b], p.uz[b], p.cos_variant);
    c = fmin(1.0, fmax(-1.0, c));
    const double ch = __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(1.0, c)));
    const double sh = __dsqrt_rn(__dmul_rn(0.5, __dsub_rn(1.0, c)));
    const double om1 = p.omega[a], om2 = p.omega[b];
    const double odl2b = p.odl2[b];
    const double io1 = p.odl2[a] > 0.0 ? 1.0 / p.odl2[a] : 0.0;
    const double io2 = p.odl2[b] > 0.0 ? 1.0 / p.odl2[b] : 0.0;
    const bool srt = p.sorted[a] && p.sorted[b];
    const int64_t A0 = p.pstart[a], B0 = p.pstart[b];
    // pixels, and the weights of their column products: an f1 pixel i enters
    // with w_i/Om2 (S) and w_i/O2 (L), an f2 pixel j with w_j/Om1 and w_j/O1
    const double kS1 = 1.0 / om2, kS2 = 1.0 / om1;
    for (int k = tid; k < L1; k += DT) {
      const double4 q = p.pix8[A0 + k];
      sd[k] = q.x; sw[k] = q.y; sl[k] = p.dl[A0 + k];
      ksc[k] = q.y * kS1; klc[k] = q.y * io2;
    }
    for (int k = tid; k < L2; k += DT) {
      const double4 q = p.pix8[B0 + k];
      sd[ML + k] = q.x; sw[ML + k] = q.y; sl[ML + k] = p.dl[B0 + k];
      ksc[ML + k] = q.y * kS2; klc[ML + k] = q.y * io1;
    }
    if (tid == 0) { s_T0 = INT_MAX; s_T1 = -1; s_maxspan = 0; }
    __syncthreads();
    // ---- phase 1: columns, one warp per pixel: side 0 = f1 pixels (partners in
    // f2), side 1 = f2 pixels (partners in f1); built in shared memory with the
    // lanes over the partners, then stored to the CTA's scratch
    for (int side = 0; side < 2; ++side) {
      const int Lm = side == 0 ? L1 : L2, Lo = side == 0 ? L2 : L1;
      const double* dm = sd + side * ML;
      const double* dO = sd + (1 - side) * ML;
      const double* wO = sw + (1 - side) * ML;
      const double* lO = sl + (1 - side) * ML;
      double* cS = colS + (size_t)side * ML * TS * NS;
      double* cL = colL + (size_t)side * ML * TS * NS;
      for (int m = warp; m < Lm; m += NW) {
        const double d = dm[m];
        int jlo = 0, jhi = Lo;
        if (srt) {   // partners with |d - d'| ch <= rpmax and (d + d') sh <= rtmax (+ margin)
          const double reach = ch > 0.0 ? ((double)np + 1e-3) / (ch * p.binner_rp) : 1e300;
          const double rt_reach = sh > 0.0 ? ((double)nt + 1e-3) / (sh * p.binner_rt) : 1e300;
          const double tl = d - reach - 1e-6 * fabs(d) - 1e-6;
          const double th = fmin(d + reach, rt_reach - d) + 1e-6 * fabs(d) + 1e-6;
          jlo = warp_first(dO, 0, Lo, [&](double v) { return v > tl; });
          jhi = warp_first(dO, jlo, Lo, [&](double v) { return !(v < th); });
        }
        // window of rt bins the column can touch, and the built rows
        int wlo = 0, nrow = 0;
        int lo = INT_MAX, hi = -1;
        if (srt) {
          // sorted: the rt bin is non-decreasing in the partner index, so the
          // partners at the two ends of the range bound the window; one pass,
          // each lane over a contiguous segment of partners, equal-bin runs
          // merged in registers before the shared-memory add
          if (jlo < jhi) {
            const double f0 = side == 0 ? pair_ft(d, dO[jlo], sh, p) : pair_ft(dO[jlo], d, sh, p);
            const double f1v = side == 0 ? pair_ft(d, dO[jhi - 1], sh, p) : pair_ft(dO[jhi - 1], d, sh, p);
            const double flo = fmax(f0, 0.0), fhi = fmin(f1v, (double)(nt - 1));
            if (flo <= fhi) {
              wlo = (int)flo;
              nrow = (int)fhi - wlo + 1;
            }
          }
          if (nrow > TSB) {
            if (lane == 0) atomicAdd(p.err, 1ull);
            nrow = 0;
          }
          if (nrow > 0) {
            if ((np & 1) == 0) {   // 16-byte stores (both builders start on 16 bytes for even np)
              double2* s2 = reinterpret_cast<double2*>(myS);
              double2* l2 = reinterpret_cast<double2*>(myL);
              for (int q = lane; q < nrow * np / 2; q += 32) { s2[q] = make_double2(0.0, 0.0); l2[q] = make_double2(0.0, 0.0); }
            } else {
              for (int q = lane; q < nrow * np; q += 32) { myS[q] = 0.0; myL[q] = 0.0; }
            }
            __syncwarp();
            const int cnt = jhi - jlo, seg = (cnt + 31) / 32;
            int j = jlo + lane * seg;
            const int je = min(jhi, j + seg);
            int cbp = -1, cbt = -1;
            double as = 0.0, al = 0.0;
            auto merge = [&](bool in, int bp, int bt, double wj, double lj) {
              if (!in) { bp = -1; bt = -1; }
              if (bp != cbp || bt != cbt) {
                if (cbp >= 0) {
                  const int q = (cbt - wlo) * np + cbp;
                  atomicAdd(&myS[q], as);
                  atomicAdd(&myL[q], al);
                }
                cbp = bp; cbt = bt; as = 0.0; al = 0.0;
              }
              if (in) {
                as += wj;
                al = fma(wj, lj, al);
                lo = min(lo, bt);
                hi = max(hi, bt);
              }
            };
            // bins of four partners at a time (independent FP64 chains), then
            // the runs in partner order
            for (; j + 4 <= je; j += 4) {
              int bp[4], bt[4];
              bool in[4];
              double wj[4], lj[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const double dj = dO[j + u];
                wj[u] = wO[j + u];
                lj[u] = lO[j + u];
                in[u] = side == 0 ? pair_bin2(d, dj, ch, sh, p, bp[u], bt[u]) : pair_bin2(dj, d, ch, sh, p, bp[u], bt[u]);
              }
#pragma unroll
              for (int u = 0; u < 4; ++u) merge(in[u], bp[u], bt[u], wj[u], lj[u]);
            }
            for (; j < je; ++j) {
              int bp, bt;
              const bool in = side == 0 ? pair_bin2(d, dO[j], ch, sh, p, bp, bt) : pair_bin2(dO[j], d, ch, sh, p, bp, bt);
              merge(in, bp, bt, wO[j], lO[j]);
            }
            if (cbp >= 0) {
              const int q = (cbt - wlo) * np + cbp;
              atomicAdd(&myS[q], as);
              atomicAdd(&myL[q], al);
            }
          }
          for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
          }
        } else {
          // unsorted: a first pass finds the rt bins the column touches
          for (int o = jlo + lane; o < jhi; o += 32) {
            int bp, bt;
            const bool in = side == 0 ? pair_bin2(d, dO[o], ch, sh, p, bp, bt) : pair_bin2(dO[o], d, ch, sh, p, bp, bt);
            if (in) { lo = min(lo, bt); hi = max(hi, bt); }
          }
          for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
          }
          if (hi >= lo && hi - lo + 1 <= TS) {
            wlo = lo;
            nrow = hi - lo + 1;
            for (int q = lane; q < nrow * np; q += 32) { myS[q] = 0.0; myL[q] = 0.0; }
            __syncwarp();
            for (int o = jlo + lane; o < jhi; o += 32) {
              int bp, bt;
              const bool in = side == 0 ? pair_bin2(d, dO[o], ch, sh, p, bp, bt) : pair_bin2(dO[o], d, ch, sh, p, bp, bt);
              if (in) {
                const int q = (bt - wlo) * np + bp;
                atomicAdd(&myS[q], wO[o]);
                atomicAdd(&myL[q], wO[o] * lO[o]);
              }
            }
          }
        }
        int sp = hi >= lo ? hi - lo + 1 : 0;
        if (sp > TS) {
          if (lane == 0) atomicAdd(p.err, 1ull);
          sp = 0;
        }
        if (lane == 0) {
          tlo[side * ML + m] = lo;
          span[side * ML + m] = sp;
        }
        __syncwarp();
        if (sp > 0) {
          // rows lo..hi of the built window go to the CTA's scratch
          double* rs = cS + (size_t)m * TS * NS;
          double* rl = cL + (size_t)m * TS * NS;
          const int off = (lo - wlo) * np;
          if ((np & 1) == 0) {   // NS == np: 16-byte copies, every row start on 16 bytes
            const int h = np / 2;
            for (int row = 0; row < sp; ++row) {
              const double2* ss = reinterpret_cast<const double2*>(myS + off + row * np);
              const double2* sl2 = reinterpret_cast<const double2*>(myL + off + row * np);
              double2* ds = reinterpret_cast<double2*>(rs + row * NS);
              double2* dl = reinterpret_cast<double2*>(rl + row * NS);
              for (int c2 = lane; c2 < h; c2 += 32) { ds[c2] = ss[c2]; dl[c2] = sl2[c2]; }
            }
          } else {
            for (int row = 0; row < sp; ++row) {
              for (int col = lane; col < NS; col += 32) {
                rs[row * NS + col] = col < np ? myS[off + row * np + col] : 0.0;
                rl[row * NS + col] = col < np ? myL[off + row * np + col] : 0.0;
              }
            }
          }
          if (lane == 0) {
            atomicMin(&s_T0, lo);
            atomicMax(&s_T1, lo + sp - 1);
            atomicMax(&s_maxspan, sp);
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    const int T0 = s_T0, T1 = s_T1, maxspan = s_maxspan;
    if (T1 < T0) {   // no pixel pair in range
      __syncthreads();
      continue;
    }
    for (int e = tid; e < 4 * nt * np; e += DT) {
      const int tb = (e / np) % nt;
      if (tb >= T0 && tb <= T1) mom[e] = 0.0;
    }
    __syncthreads();
    const double cA = 1.0 / (om1 * om2), cB = io2 / om1, cC = io1 / om2, cD = io1 * io2;
    // ---- phase 2: blocks (t, u), T0 <= t <= u <= T1, diagonal blocks first.
    // The rows of a chunk of pixels are copied from the column scratch into
    // shared memory asynchronously (16-byte cp.async, no registers), one chunk
    // ahead of the chunk the MMA warps multiply (double buffering); the row
    // weights k_S, k_L scale the A fragments as the MMA warps read them.
    const int nT = T1 - T0 + 1;
    const int nblk = nT + nT * (nT - 1) / 2;
    const int SET = CH * NPAD;   // doubles of one row set
    for (int kb = 0; kb < nblk; ++kb) {
      int t, u;
      if (kb < nT) { t = u = T0 + kb; }
      else {   // off-diagonal pairs in row-major order of the upper triangle
        int r = kb - nT, tt = 0;
        while (r >= nT - 1 - tt) { r -= nT - 1 - tt; ++tt; }
        t = T0 + tt; u = t + 1 + r;
      }
      const bool diag = t == u;
      double acc[CC][4];
#pragma unroll
      for (int c = 0; c < CC; ++c) { acc[c][0] = 0.0; acc[c][1] = 0.0; acc[c][2] = 0.0; acc[c][3] = 0.0; }
      if (u - t < maxspan) {
        // pixels whose column spans both t and u
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        for (int side = 0; side < 2; ++side) {
          const int Lm = side == 0 ? L1 : L2;
          for (int m = tid; m < Lm; m += DT) {
            const int lo = tlo[side * ML + m], sp = span[side * ML + m];
            if (sp > 0 && lo <= t && u < lo + sp) {
              const int x = atomicAdd(&s_cnt, 1);
              plist[x] = (side << 16) | m;
              if (p.row_offsets) roff[x] = ((side * ML + m) * TS + t - lo) * NS;   // row u is (u - t) NS further
            }
          }
        }
        __syncthreads();
        const int n = s_cnt;
        const int nch = (n + CH - 1) / CH;
        // issue the copies of chunk ci into buffer ci & 1 (rows beyond the
        // chunk are zeroed with plain stores).  Columns NS .. NPAD-1 are not
        // copied: they keep older contents, which reach only accumulator
        // entries that are never flushed (tile columns >= np), except the
        // moment columns NS .. NS+3 written below for the A rows of a
        // diagonal block
        auto issue = [&](int ci) {
          double* buf = stage + (size_t)(ci & 1) * 4 * SET;
          double* kb2 = kbuf + (size_t)(ci & 1) * 4 * CH;
          const int c0 = ci * CH, rows = min(CH, n - c0), rows8 = (rows + 7) & ~7;
          const int nset = diag ? 2 : 4;           // a diagonal block reads the rows of t only
          const int segs = NS / 2;                 // 16-byte segments of a row
          // q = (set CH + r) segs + sg over whole chunks; rows r >= rows are skipped
          for (int q = tid; q < nset * CH * segs; q += DT) {
            const int sr = (int)__umulhi((unsigned)q, seg_magic), sg = q - sr * segs;
            const int set = sr / CH, r = sr - set * CH;
            if (r >= rows) continue;
            const double* colb = (set & 1) ? colL : colS;
            const double* src;
            if (p.row_offsets) {
              src = colb + roff[c0 + r] + (set < 2 ? 0 : (u - t) * NS) + 2 * sg;
            } else {
              const int pk = plist[c0 + r], side = pk >> 16, m = pk & 0xffff;
              const int lo = tlo[side * ML + m];
              const int bin = set < 2 ? t : u;
              src = colb + (size_t)side * ML * TS * NS + ((size_t)m * TS + (bin - lo)) * NS + 2 * sg;
            }
            __pipeline_memcpy_async(buf + (size_t)set * SET + (size_t)r * NPAD + 2 * sg, src, 16);
          }
          for (int q = tid; q < nset * (rows8 - rows) * NPAD; q += DT) {
            const int set = q / ((rows8 - rows) * NPAD), rem = q - set * (rows8 - rows) * NPAD;
            buf[(size_t)set * SET + (size_t)rows * NPAD + rem] = 0.0;
          }
          for (int r = tid - (DT - 32); r >= 0 && r < rows8; r += 32) {   // the last warp
            double ks = 0.0, kl = 0.0, w0 = 0.0, w1 = 0.0;
            if (r < rows) {
              const int pk = plist[c0 + r], side = pk >> 16, m = pk & 0xffff;
              ks = ksc[side * ML + m];
              kl = klc[side * ML + m];
              if (side == 0) { w0 = sw[m]; w1 = sw[m] * sl[m]; }
            }
            kb2[r] = ks;
            kb2[CH + r] = kl;
            kb2[2 * CH + r] = w0;
            kb2[3 * CH + r] = w1;
            if (diag && NS + 4 <= 64) {   // moment columns of the S and L rows of bin t
              double dlm = 0.0;
              bool f1r = false;
              if (r < rows) {
                const int pk = plist[c0 + r];
                f1r = (pk >> 16) == 0;
                dlm = sl[pk & 0xffff];
              }
              double* rs = buf + (size_t)r * NPAD + NS;
              double* rl = buf + SET + (size_t)r * NPAD + NS;
              rs[0] = f1r ? om2 : 0.0; rs[1] = f1r ? om2 * dlm : 0.0; rs[2] = 0.0; rs[3] = 0.0;
              rl[0] = 0.0; rl[1] = 0.0; rl[2] = f1r ? odl2b : 0.0; rl[3] = f1r ? odl2b * dlm : 0.0;
            }
          }
          __pipeline_commit();
        };
        if (nch > 0) issue(0);
        for (int ci = 0; ci < nch; ++ci) {
          if (ci + 1 < nch) {
            issue(ci + 1);
            __pipeline_wait_prior(1);   // this thread's copies of chunk ci have landed
          } else {
            __pipeline_wait_prior(0);
          }
          __syncthreads();               // everyone's copies of chunk ci have landed
          const double* buf = stage + (size_t)(ci & 1) * 4 * SET;
          const double* kb2 = kbuf + (size_t)(ci & 1) * 4 * CH;
          const double* SA = buf;                      // rows of bin t: S, L (unscaled)
          const double* LA = buf + SET;
          const double* SB = diag ? SA : buf + 2 * SET;   // rows of bin u
          const double* LB = diag ? LA : buf + 3 * SET;
          const int c0 = ci * CH, rows = min(CH, n - c0), rows8 = (rows + 7) & ~7;
          if (tid == 0) n_mma += (unsigned long long)((rows + 3) / 4) * ntile * ntile * 2;
          if (diag && !(NS + 4 <= 64)) {   // moments of bin t from the rows of the f1 pixels
            for (int e = tid; e < 4 * np; e += DT) {
              const int q = e / np, bq = e - q * np;
              const double* src = (q < 2 ? SA : LA) + bq;   // 0: M0, 1: Mi from S; 2: Mj, 3: Mij from L
              const double* cw = kb2 + ((q == 0 || q == 2) ? 2 : 3) * CH;   // f1 w or w dl, 0 for f2 rows
              double sacc = 0.0;
#pragma unroll 4
              for (int r = 0; r < rows; ++r) sacc = fma(cw[r], src[r * NPAD], sacc);
              mom[(q * nt + t) * np + bq] += sacc;
            }
          }
          {
            const int bp0 = 16 * mt + grp, bp1 = bp0 + 8;
            const int arows = (diag && NS + 4 <= 64) ? NS + 4 : np;   // A rows NS..NS+3: the moments
            const bool v0 = bp0 < arows, v1 = bp1 < arows;
            for (int r0 = 0; r0 < rows8; r0 += 8) {
              const int ra = (r0 + kq) * NPAD, rb = ra + 4 * NPAD;
              const double ks0 = kb2[r0 + kq], ks1 = kb2[r0 + kq + 4];
              const double kl0 = kb2[CH + r0 + kq], kl1 = kb2[CH + r0 + kq + 4];
              const double as0 = v0 ? SA[ra + bp0] * ks0 : 0.0, as1 = v1 ? SA[ra + bp1] * ks0 : 0.0;
              const double as2 = v0 ? SA[rb + bp0] * ks1 : 0.0, as3 = v1 ? SA[rb + bp1] * ks1 : 0.0;
              const double al0 = v0 ? LA[ra + bp0] * kl0 : 0.0, al1 = v1 ? LA[ra + bp1] * kl0 : 0.0;
              const double al2 = v0 ? LA[rb + bp0] * kl1 : 0.0, al3 = v1 ? LA[rb + bp1] * kl1 : 0.0;
#pragma unroll
              for (int c = 0; c < CC; ++c) {
                const int nt8 = ng + nwm * c;
                if (nt8 < ntile) {
                  lya_dmma_16x8x8(acc[c], as0, as1, as2, as3, SB[ra + 8 * nt8 + grp], SB[rb + 8 * nt8 + grp]);
                  lya_dmma_16x8x8(acc[c], al0, al1, al2, al3, LB[ra + 8 * nt8 + grp], LB[rb + 8 * nt8 + grp]);
                }
              }
            }
          }
          __syncthreads();               // buffer ci & 1 is free for chunk ci + 2
        }
        if (diag && NS + 4 <= 64) {   // accumulator rows NS..NS+3: the moments of bin t
#pragma unroll
          for (int h2 = 0; h2 < 2; ++h2) {
            const int q = 16 * mt + grp + 8 * h2 - NS;
            if (q >= 0 && q < 4) {
#pragma unroll
              for (int c = 0; c < CC; ++c) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                  const int nt8 = ng + nwm * c, bq = 8 * nt8 + 2 * kq + i;
                  if (nt8 < ntile && bq < np) mom[(q * nt + t) * np + bq] = acc[c][2 * h2 + i];
                }
              }
            }
          }
          __syncthreads();
        }
      }
      // flush: column products (subtracted), rank-4 part, diagonal; warp
      // (trow, thalf) writes the entries (8 trow + grp, 8c + 2kq + i) of its columns
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {
        const int bp = 16 * mt + grp + 8 * h2;
        if (bp < np) {
          const double* mtp = mom + (size_t)t * np + bp;   // + q*nt*np
          const double m0a = mtp[0], mia = mtp[nt * np], mja = mtp[2 * nt * np], mija = mtp[3 * nt * np];
#pragma unroll
          for (int c = 0; c < CC; ++c) {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int nt8 = ng + nwm * c;
              const int bq = 8 * nt8 + 2 * kq + i;
              if (nt8 >= ntile || bq >= np) continue;
              const double* mu = mom + (size_t)u * np + bq;
              double v = m0a * mu[0] * cA + mja * mu[2 * nt * np] * cB + mia * mu[nt * np] * cC +
                         mija * mu[3 * nt * np] * cD - acc[c][2 * h2 + i];
              const int A = bp * nt + t, B = bq * nt + u;
              if (A == B) {
                v += m0a;
                if (m0a != 0.0) atomicAdd(&p.W[A], m0a);
              }
              if (v != 0.0) {
                atomicAdd(&p.D[(size_t)A * nb + B], v);
                if (t != u) atomicAdd(&p.D[(size_t)B * nb + A], v);
              }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0 && n_mma) atomicAdd(p.mma, n_mma);
}

template <int V>
cudaError_t set_dist_smem_v(int smem) {
  return cudaFuncSetAttribute(k_dist<DIST_SHAPES[V].dt, DIST_SHAPES[V].ch>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              smem);
}

cudaError_t set_dist_smem(int shape, int smem) {
  switch (shape) {
    case 1: return set_dist_smem_v<1>(smem);
    case 2: return set_dist_smem_v<2>(smem);
    case 3: return set_dist_smem_v<3>(smem);
    case 4: return set_dist_smem_v<4>(smem);
    default: return set_dist_smem_v<0>(smem);
  }
}

template <int V>
cudaError_t launch_dist_v(int grid, size_t smem, cudaStream_t s, const DistParams& p) {
  k_dist<DIST_SHAPES[V].dt, DIST_SHAPES[V].ch><<<grid, DIST_SHAPES[V].dt, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_dist(int shape, int grid, size_t smem, cudaStream_t s, const DistParams& p) {
  switch (shape) {
    case 1: return launch_dist_v<1>(grid, smem, s, p);
    case 2: return launch_dist_v<2>(grid, smem, s, p);
    case 3: return launch_dist_v<3>(grid, smem, s, p);
    case 4: return launch_dist_v<4>(grid, smem, s, p);
    default: return launch_dist_v<0>(grid, smem, s, p);
  }
}
static_assert(N_DIST_SHAPES == 5, "the launch tables above cover every shape");
static_assert(DIST_SHAPES[0].ch % 8 == 0 && DIST_SHAPES[1].ch % 8 == 0 && DIST_SHAPES[2].ch % 8 == 0 &&
                  DIST_SHAPES[3].ch % 8 == 0 && DIST_SHAPES[4].ch % 8 == 0 && DIST_SHAPES[3].dt % 128 == 0,
              "chunks hold whole MMA K steps; the warps cover the four tile rows");

}  // namespace

extern "C" int lya_dist_config(lya_ctx* ctx, int32_t shape, int64_t max_items) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_dist_config: ctx is NULL");
  if (shape < 0 || shape >= N_DIST_SHAPES)
    return lya_fail(ctx, LYA_ERR_ARG, "lya_dist_config: shape %d outside [0,%d)", shape, N_DIST_SHAPES);
  if (max_items < 0) return lya_fail(ctx, LYA_ERR_ARG, "lya_dist_config: max_items < 0");
  ctx->dist_shape = shape;
  ctx->dist_max_items = max_items;
  return LYA_OK;
}

extern "C" int lya_dist_run(lya_ctx* ctx, double* D, double* W) {
  if (!ctx) return lya_fail(nullptr, LYA_ERR_ARG, "lya_dist_run: ctx is NULL");
  if (!ctx->bins_set) return lya_fail(ctx, LYA_ERR_STATE, "lya_dist_run: call lya_set_bins first");
  if (ctx->cat.n == 0) return lya_fail(ctx, LYA_ERR_STATE, "lya_dist_run: no forests uploaded");
  if (!ctx->cat.has_dl || !ctx->cat.has_moments)
    return lya_fail(ctx, LYA_ERR_STATE, "lya_dist_run: upload dl, omega and odl2 with the forests");
  const int np = ctx->np, nt = ctx->nt, nb = np * nt;
  if (np > NP_MAX) return lya_fail(ctx, LYA_ERR_ARG, "lya_dist_run: np = %d above %d r_par bins", np, NP_MAX);
  LYA_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
  int max_len = 1;
  for (int64_t f = 0; f < ctx->cat.n; ++f)
    max_len = std::max<int>(max_len, (int)(ctx->h_start[f + 1] - ctx->h_start[f]));
  if (max_len > 65535) return lya_fail(ctx, LYA_ERR_DATA, "lya_dist_run: forests longer than 65535 pixels");
  const int npad = stage_npad(np);
  const int shape = ctx->dist_shape;
  const int DT = DIST_SHAPES[shape].dt, CH = DIST_SHAPES[shape].ch, NW = DT / 32;
  const size_t stage_len = (size_t)stage_doubles(CH, NW, np);
  const size_t smem = sizeof(double) * (10 * (size_t)max_len + stage_len + 8 * (size_t)CH) +
                      sizeof(int) * (6 * (size_t)max_len);
  if (smem > 227 * 1024)
    return lya_fail(ctx, LYA_ERR_DATA, "lya_dist_run: forests of %d pixels need %zu B of shared memory (shape %d)",
                    max_len, smem, shape);
  const int grid = ctx->num_sms;
  // scratch and outputs kept in the context, so later calls (one per healpix
  // pixel in the drop-in driver) allocate nothing and replay the captured graph
  DistScratch& ds = ctx->dist;
  if (!ds.D || ds.nb != nb || ds.max_len < max_len || ds.grid != grid) {
    lya_free(ds.D); lya_free(ds.W); lya_free(ds.col); lya_free(ds.mom); lya_free(ds.err);
    if (ds.graph) { cudaGraphExecDestroy(ds.graph); ds.graph = nullptr; }
    ds = DistScratch{};
    cudaError_t e = lya_alloc(&ds.D, (size_t)nb * nb);
    if (e == cudaSuccess) e = lya_alloc(&ds.W, nb);
    if (e == cudaSuccess) e = lya_alloc(&ds.col, (size_t)grid * 2 * 2 * max_len * TS * col_stride(np));
    if (e == cudaSuccess) e = lya_alloc(&ds.mom, (size_t)grid * 4 * nt * np);
    if (e == cudaSuccess) e = lya_alloc(&ds.err, 4);
    if (e != cudaSuccess) {
      lya_free(ds.D); lya_free(ds.W); lya_free(ds.col); lya_free(ds.mom); lya_free(ds.err);
      ds = DistScratch{};
      return lya_fail(ctx, LYA_ERR_ALLOC, "lya_dist_run: device allocation failed");
    }
    ds.nb = nb; ds.max_len = max_len; ds.grid = grid;
  }
  cudaStream_t s = ctx->stream;
  const long long n_items = ctx->dist_max_items > 0 ? std::min<long long>(ctx->wq.n_pairs, ctx->dist_max_items)
                                                    : ctx->wq.n_pairs;
  DistParams p;
  memset(&p, 0, sizeof(p));   // padding bytes take part in the graph key
  p.pix8 = ctx->cat.pix8; p.dl = ctx->cat.dl; p.pstart = ctx->cat.pstart; p.len = ctx->cat.len;
  p.sorted = ctx->cat.sorted; p.ux = ctx->cat.ux; p.uy = ctx->cat.uy; p.uz = ctx->cat.uz;
  p.omega = ctx->cat.omega; p.odl2 = ctx->cat.odl2; p.f1 = ctx->wq.f1; p.f2 = ctx->wq.f2;
  p.n_items = reinterpret_cast<const long long*>(ds.err + 2); p.max_len = ds.max_len;
  p.binner_rp = (double)np / ctx->rpmax; p.binner_rt = (double)nt / ctx->rtmax;
  p.np = np; p.nt = nt; p.nb = nb; p.cos_variant = ctx->cos_variant; p.npad = npad;
  p.col = ds.col; p.moments = ds.mom; p.D = ds.D; p.W = ds.W; p.err = ds.err; p.next = ds.err + 1;
  p.mma = ds.err + 3;
  p.shape = shape;
  size_t smem_run = sizeof(double) * (10 * (size_t)ds.max_len + stage_len + 8 * (size_t)CH) +
                    sizeof(int) * (6 * (size_t)ds.max_len);
  // the pixel list's row offsets (one int per listed pixel) when shared memory has room
  if (smem_run + sizeof(int) * 2 * (size_t)ds.max_len <= 227 * 1024) {
    smem_run += sizeof(int) * 2 * (size_t)ds.max_len;
    p.row_offsets = 1;
  }
  static_assert(sizeof(DistParams) <= sizeof(ds.key), "graph key does not fit");
  cudaError_t e = cudaSuccess;
  if (!ds.graph || memcmp(ds.key, &p, sizeof(p)) != 0) {
    if (ds.graph) { cudaGraphExecDestroy(ds.graph); ds.graph = nullptr; }
    e = set_dist_smem(shape, (int)smem_run);
    cudaGraph_t g = nullptr;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t eq = cudaMemsetAsync(ds.D, 0, sizeof(double) * (size_t)nb * nb, s);
      if (eq == cudaSuccess) eq = cudaMemsetAsync(ds.W, 0, sizeof(double) * nb, s);
      if (eq == cudaSuccess) eq = cudaMemsetAsync(ds.err, 0, 2 * sizeof(unsigned long long), s);
      if (eq == cudaSuccess) eq = cudaMemsetAsync(ds.err + 3, 0, sizeof(unsigned long long), s);
      if (eq == cudaSuccess) {
        eq = launch_dist(shape, grid, smem_run, s, p);
      }
      const cudaError_t ec = cudaStreamEndCapture(s, &g);
      e = eq != cudaSuccess ? eq : ec;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ds.graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ds.graph = nullptr;
      return lya_fail(ctx, LYA_ERR_CUDA, "lya_dist_run: capture: %s", cudaGetErrorString(e));
    }
    memcpy(ds.key, &p, sizeof(p));
  }
  e = cudaMemcpyAsync(ds.err + 2, &n_items, sizeof(n_items), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
  if (e == cudaSuccess) e = cudaGraphLaunch(ds.graph, s);
  if (e == cudaSuccess) {
    ctx->launches++;
    e = cudaEventRecord(ctx->ev1, s);
  }
  unsigned long long nerr = 0, nmma = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nerr, ds.err, sizeof(nerr), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nmma, ds.err + 3, sizeof(nmma), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && D) e = cudaMemcpyAsync(D, ds.D, sizeof(double) * (size_t)nb * nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && W) e = cudaMemcpyAsync(W, ds.W, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (e != cudaSuccess) return lya_fail(ctx, LYA_ERR_CUDA, "lya_dist_run: %s", cudaGetErrorString(e));
  ctx->last.kernel_ms = ms;
  ctx->last.dist_mma_flops = (double)nmma * 2.0 * 8 * 8 * 4;   // m8n8k4: 256 FMA per MMA
  if (nerr) return lya_fail(ctx, LYA_ERR_DATA, "lya_dist_run: %llu pixels pair into more than %d rt bins", nerr, TS);
  return LYA_OK;
}
