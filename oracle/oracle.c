/*
 * CPU oracle for the lya2pcf pair-binning path.  TEST INFRASTRUCTURE ONLY: the
 * tests, the smoke check and the CPU-baseline leg of the benchmark call it as a
 * checker; no product code path links or calls it.
 *
 * Plain FP64 restatement of the reference algorithms, one function per
 * reference routine, written for clarity rather than speed (the only
 * concession to speed is a thread pool over owner pixels):
 *
 *   orc_neighbours_*   forest_class.py:78-98 (quasar.neighborhood): keep f2 when
 *                      ((x1*x2 + y1*y2) + z1*z2) > cos(angmax), name1 != name2 and
 *                      ra1 < ra2, evaluated in Python's operation order; output
 *                      order = ascending caller-supplied key (healpix pixel, then
 *                      position inside the pixel), the order query_disc +
 *                      list iteration produce.
 *   orc_corr           cuda_kernels.cpp:90-162 (pair_correlation) driven as
 *                      correlation_procedures_pycuda.py:141-166 drives it: for
 *                      every listed forest pair and every pixel pair,
 *                        cos12 = x1*x2 + y1*y2 + z1*z2   (contraction order: see
 *                                                         orc_cos12)
 *                        ch = sqrt(0.5*(1+cos12)), sh = sqrt(0.5*(1-cos12))
 *                        rp = |dc1-dc2|*ch,  rt = (dc1+dc2)*sh
 *                        bp = floor(rp*np/rpmax), bt = floor(rt*nt/rtmax)
 *                        in range (0 <= bp < np, 0 <= bt < nt):
 *                          W += w1*w2, DW += dw1*dw2
 *                      plus the new outputs: N (count), RP = sum w1w2*rp,
 *                      RT = sum w1w2*rt, Z = sum w1w2*(z1+z2)/2, and DWABS =
 *                      sum |dw1*dw2| (the condition scale of DW, oracle only).
 *                      mode ORC_CPU_FORMULA instead restates the numba kernel
 *                      correlation_procedures_cpu.py:46-84 (ra/dec angle with the
 *                      2-arcsec small-angle branch, the dtheta < angmax cut and
 *                      int(r/rmax*n) truncation).
 *   orc_corr_wdw       the reference kernel's own work only (W and DW with the
 *                      formula of orc_corr): the timed CPU baseline.
 *   orc_adjoint        gradient of L = sum_b g_b * DW_b/W_b (no reference code):
 *                      for each in-range pair in bin b,
 *                        dL/ddw_i += (g_b/W_b) dw_j,  dL/ddw_j += (g_b/W_b) dw_i,
 *                        dL/dw_i  -= (g_b xi_b/W_b) w_j, dL/dw_j -= (g_b xi_b/W_b) w_i.
 *   orc_distortion     cuda_kernels.cpp:165-278 (compute_etas, order_active,
 *                      compute_d) as distortion_procedures_pycuda.py:207-274
 *                      runs them per forest pair, in FP64 and with the FP64
 *                      binning of orc_corr.
 *   orc_distortion_mode  the same sum with a choice of pair binning:
 *                      ORC_BIN_FP64 (as orc_distortion) or ORC_BIN_FP32, the
 *                      reference distortion's own FP32 binning of
 *                      precompute_distances (cuda_kernels.cpp:67-84): FP32 dc and
 *                      unit vectors, cos in FP32, the half-angle argument
 *                      0.5*(1 +- cos) in FP64 rounded to FP32 for sqrtf,
 *                      rp = |dc1-dc2|*ch and rt = (dc1+dc2)*sh in FP32, bins by
 *                      truncation of rp*binner_rp and rt*binner_rt (FP32
 *                      binners, parameters.py:14-21 via
 *                      distortion_procedures_pycuda.py:167).
 *   orc_dist_bins      the (bin_rp, bin_rt) of every pixel pair of one forest
 *                      pair under either binning (the FP32 form is what
 *                      precompute_distances writes).
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_NQ 6 /* W, DW, RP, RT, Z, DWABS */

enum { ORC_GPU_FORMULA = 0, ORC_CPU_FORMULA = 1 };
enum { ORC_BIN_FP64 = 0, ORC_BIN_FP32 = 1 };

/* cos of the pair angle as the reference GPU kernel computes it
 * (cuda_kernels.cpp:131, "x1*x2 + y1*y2 + z1*z2" in FP64).  nvcc contracts the
 * expression with FMAs by default; the variants let the tests pin which
 * contraction the compiled reference uses.
 *   0: fma(z1,z2, fma(x1,x2, y1*y2))
 *   1: fma(z1,z2, fma(y1,y2, x1*x2))
 *   2: ((x1*x2) + (y1*y2)) + (z1*z2)   (no contraction)                      */
/* cos12 clamped to [-1, 1]: for coincident lines of sight rounding can give
 * 1 + ulp, where the reference takes the square root of a negative number
 * (cuda_kernels.cpp:132-134); the clamp gives the geometric answer rt = 0. */
static double cos12_clamped(double x1, double y1, double z1, double x2, double y2, double z2, int variant);

double orc_cos12(double x1, double y1, double z1, double x2, double y2, double z2, int variant) {
  switch (variant) {
    case 0: return fma(z1, z2, fma(x1, x2, y1 * y2));
    case 1: return fma(z1, z2, fma(y1, y2, x1 * x2));
    default: {
      double a = x1 * x2, b = y1 * y2, c = z1 * z2;
      return (a + b) + c;
    }
  }
}

static double cos12_clamped(double x1, double y1, double z1, double x2, double y2, double z2, int variant) {
  double c = orc_cos12(x1, y1, z1, x2, y2, z2, variant);
  return c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
}

/* ------------------------------------------------------------------ inputs */
typedef struct {
  int64_t n;
  const int64_t* start; /* [n+1] */
  const double* dc;
  const double* w;
  const double* dw;
  const double* z;
  const double* dl;
  const double* ux;
  const double* uy;
  const double* uz;
  const double* ra;
  const double* dec;
  const double* omega;
  const double* odl2;
} orc_forests;

/* ------------------------------------------------------------ thread pool */
typedef struct {
  void (*fn)(void* ctx, int64_t task);
  void* ctx;
  int64_t ntask;
  int64_t next;
  pthread_mutex_t mu;
} pool_t;

static void* pool_worker(void* arg) {
  pool_t* p = (pool_t*)arg;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    int64_t t = p->next++;
    pthread_mutex_unlock(&p->mu);
    if (t >= p->ntask) break;
    p->fn(p->ctx, t);
  }
  return NULL;
}

static void pool_run(int nthreads, int64_t ntask, void (*fn)(void*, int64_t), void* ctx) {
  pool_t p;
  p.fn = fn; p.ctx = ctx; p.ntask = ntask; p.next = 0;
  pthread_mutex_init(&p.mu, NULL);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  for (int i = 1; i < nthreads; ++i) pthread_create(&th[i], NULL, pool_worker, &p);
  pool_worker(&p);
  for (int i = 1; i < nthreads; ++i) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&p.mu);
}

/* ------------------------------------------------------------ neighbours */
typedef struct {
  const orc_forests* F;
  const int64_t* name;
  const int64_t* key;     /* reference visiting order of candidates */
  double angmax, mumin;
  int64_t nband;
  double band_h;
  const int64_t* band_start; /* [nband+1] into band_idx */
  const int64_t* band_idx;   /* forests sorted by (band, ra) */
  int64_t* counts;           /* [n] */
  const int64_t* offsets;    /* [n+1] or NULL (count pass) */
  int32_t* out;              /* neighbours, or NULL */
  int all_ra_in_range;
} nb_ctx;

static int cmp_key_ctx_sort(const void* a, const void* b, void* kp) {
  const int64_t* key = (const int64_t*)kp;
  int64_t ka = key[*(const int32_t*)a], kb = key[*(const int32_t*)b];
  return (ka > kb) - (ka < kb);
}

static int64_t lower_ra(const nb_ctx* c, int64_t b, double ra) {
  /* first position in band b whose ra >= ra */
  int64_t lo = c->band_start[b], hi = c->band_start[b + 1];
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (c->F->ra[c->band_idx[mid]] < ra) lo = mid + 1; else hi = mid;
  }
  return lo;
}

static inline int nb_accept(const nb_ctx* c, int64_t f1, int64_t f2) {
  const orc_forests* F = c->F;
  double a = F->ux[f1] * F->ux[f2];
  double b = F->uy[f1] * F->uy[f2];
  double d = F->uz[f1] * F->uz[f2];
  double mu = (a + b) + d;
  return mu > c->mumin && c->name[f1] != c->name[f2] && F->ra[f1] < F->ra[f2];
}

static void nb_task(void* vctx, int64_t f1) {
  nb_ctx* c = (nb_ctx*)vctx;
  const orc_forests* F = c->F;
  double dec1 = F->dec[f1], ra1 = F->ra[f1];
  int64_t b1 = (int64_t)floor((dec1 + M_PI_2) / c->band_h);
  double dlim = fabs(dec1) + c->angmax * (1.0 + 1e-6) + 1e-9;
  double dra;
  int full = !c->all_ra_in_range;
  if (dlim >= M_PI_2 - 1e-9) {
    full = 1; dra = 0.0;
  } else {
    double s = sin(0.5 * c->angmax) / cos(dlim);
    if (s >= 1.0) { full = 1; dra = 0.0; }
    else {
      dra = 2.0 * asin(s) * (1.0 + 1e-6) + 1e-9;
      if (dra >= M_PI_2) full = 1;
    }
  }
  int64_t cnt = 0;
  int32_t* dst = c->out ? c->out + c->offsets[f1] : NULL;
  for (int64_t b = b1 - 1; b <= b1 + 1; ++b) {
    if (b < 0 || b >= c->nband) continue;
    int64_t lo = c->band_start[b], hi = c->band_start[b + 1];
    if (full) {
      for (int64_t p = lo; p < hi; ++p) {
        int64_t f2 = c->band_idx[p];
        if (nb_accept(c, f1, f2)) { if (dst) dst[cnt] = (int32_t)f2; ++cnt; }
      }
      continue;
    }
    /* ra2 in (ra1, ra1 + dra]  (ra < ra2 is required) */
    int64_t p0 = lower_ra(c, b, ra1);
    for (int64_t p = p0; p < hi; ++p) {
      int64_t f2 = c->band_idx[p];
      if (F->ra[f2] > ra1 + dra) break;
      if (nb_accept(c, f1, f2)) { if (dst) dst[cnt] = (int32_t)f2; ++cnt; }
    }
    /* wrapped neighbours: ra2 in [ra1 - dra + 2pi, 2pi); disjoint from the
     * range above because dra < pi/2 here */
    if (ra1 - dra < 0.0) {
      int64_t q0 = lower_ra(c, b, ra1 - dra + 2.0 * M_PI);
      for (int64_t p = q0; p < hi; ++p) {
        int64_t f2 = c->band_idx[p];
        if (nb_accept(c, f1, f2)) { if (dst) dst[cnt] = (int32_t)f2; ++cnt; }
      }
    }
  }
  if (dst && cnt > 1) qsort_r(dst, (size_t)cnt, sizeof(int32_t), cmp_key_ctx_sort, (void*)c->key);
  c->counts[f1] = cnt;
}

typedef struct { const double* ra; const int64_t* band; } band_sort_ctx;
static int cmp_band_ra(const void* a, const void* b, void* vp) {
  const band_sort_ctx* s = (const band_sort_ctx*)vp;
  int64_t ia = *(const int64_t*)a, ib = *(const int64_t*)b;
  if (s->band[ia] != s->band[ib]) return (s->band[ia] > s->band[ib]) - (s->band[ia] < s->band[ib]);
  if (s->ra[ia] != s->ra[ib]) return (s->ra[ia] > s->ra[ib]) - (s->ra[ia] < s->ra[ib]);
  return (ia > ib) - (ia < ib);
}

/* Neighbour lists of every forest.  Call with out == NULL to get counts[n],
 * then with offsets (exclusive scan of counts, [n+1]) and out[offsets[n]]. */
int orc_neighbours(const orc_forests* F, const int64_t* name, const int64_t* key, double angmax, double mumin,
                   int64_t* counts, const int64_t* offsets, int32_t* out, int nthreads) {
  int64_t n = F->n;
  double h = angmax * (1.0 + 1e-6) + 1e-9;
  int64_t nband = (int64_t)ceil(M_PI / h) + 2;
  int64_t* band = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t* bstart = (int64_t*)calloc((size_t)nband + 1, sizeof(int64_t));
  if (!band || !idx || !bstart) { free(band); free(idx); free(bstart); return -1; }
  int all_in = 1;
  for (int64_t f = 0; f < n; ++f) {
    int64_t b = (int64_t)floor((F->dec[f] + M_PI_2) / h);
    if (b < 0) b = 0;
    if (b >= nband) b = nband - 1;
    band[f] = b;
    idx[f] = f;
    if (!(F->ra[f] >= 0.0 && F->ra[f] < 2.0 * M_PI)) all_in = 0;
  }
  band_sort_ctx bs = {F->ra, band};
  qsort_r(idx, (size_t)n, sizeof(int64_t), cmp_band_ra, &bs);
  for (int64_t f = 0; f < n; ++f) bstart[band[f] + 1]++;
  for (int64_t b = 0; b < nband; ++b) bstart[b + 1] += bstart[b];
  nb_ctx c;
  c.F = F; c.name = name; c.key = key; c.angmax = angmax; c.mumin = mumin;
  c.nband = nband; c.band_h = h; c.band_start = bstart; c.band_idx = idx;
  c.counts = counts; c.offsets = offsets; c.out = out; c.all_ra_in_range = all_in;
  pool_run(nthreads, n, nb_task, &c);
  free(band); free(idx); free(bstart);
  return 0;
}

/* ------------------------------------------------------------ correlation */
typedef struct {
  const orc_forests* F;
  const int32_t* f1;
  const int32_t* f2;
  const int64_t* slot_item_start; /* [nslot+1] item ranges per output slot */
  double rpmax, rtmax;
  int np, nt;
  int mode, cos_variant;
  double angmax;
  double* out;      /* [nslot][ORC_NQ][np*nt] */
  uint64_t* cnt;    /* [nslot][np*nt] */
} corr_ctx;

/* numba kernel constants (parameters.py:38) */
static const double CHIQUITO = 2. / 3600. * 3.14159 / 180.;

static void corr_pair(const corr_ctx* c, int64_t a, int64_t b, double* h, uint64_t* n) {
  const orc_forests* F = c->F;
  const int nb = c->np * c->nt;
  int64_t s1 = F->start[a], l1 = F->start[a + 1] - s1;
  int64_t s2 = F->start[b], l2 = F->start[b + 1] - s2;
  double chh, shh;
  if (c->mode == ORC_GPU_FORMULA) {
    double cos12 = cos12_clamped(F->ux[a], F->uy[a], F->uz[a], F->ux[b], F->uy[b], F->uz[b], c->cos_variant);
    chh = sqrt(0.5 * (1. + cos12));
    shh = sqrt(0.5 * (1. - cos12));
  } else {
    double ra1 = F->ra[a], dec1 = F->dec[a], ra2 = F->ra[b], dec2 = F->dec[b];
    double dth;
    if (fabs(ra1 - ra2) < CHIQUITO && fabs(dec1 - dec2) < CHIQUITO) {
      double t1 = (ra1 - ra2) * cos(dec1), t2 = dec1 - dec2;
      dth = sqrt(t1 * t1 + t2 * t2);
    } else {
      double t1 = sin(dec1) * sin(dec2), t2 = cos(dec1) * cos(dec2) * cos(ra1 - ra2);
      dth = acos(t1 + t2);
    }
    chh = cos(0.5 * dth);
    shh = sin(0.5 * dth);
    if (!(dth < c->angmax)) return;
  }
  const double binner_rp = (double)c->np / c->rpmax;
  const double binner_rt = (double)c->nt / c->rtmax;
  for (int64_t i = 0; i < l1; ++i) {
    double d1 = F->dc[s1 + i], w1 = F->w[s1 + i], dw1 = F->dw[s1 + i], z1 = F->z[s1 + i];
    for (int64_t j = 0; j < l2; ++j) {
      double d2 = F->dc[s2 + j];
      double rp = fabs(d1 - d2) * chh;
      double rt = (d1 + d2) * shh;
      int bp, bt;
      if (c->mode == ORC_GPU_FORMULA) {
        double fp = floor(rp * binner_rp), ft = floor(rt * binner_rt);
        if (!(fp >= 0.0 && fp < (double)c->np && ft >= 0.0 && ft < (double)c->nt)) continue;
        bp = (int)fp; bt = (int)ft;
      } else {
        double xp = rp / c->rpmax * c->np, xt = rt / c->rtmax * c->nt;
        if (!(xp < (double)c->np && xt < (double)c->nt && xp > -1.0 && xt > -1.0)) continue;
        bp = (int)xp; bt = (int)xt;   /* truncation, as Python int() */
      }
      int k = bp * c->nt + bt;
      double w12 = w1 * F->w[s2 + j];
      double dw12 = dw1 * F->dw[s2 + j];
      h[0 * nb + k] += w12;
      h[1 * nb + k] += dw12;
      h[2 * nb + k] += w12 * rp;
      h[3 * nb + k] += w12 * rt;
      h[4 * nb + k] += w12 * (0.5 * (z1 + F->z[s2 + j]));
      h[5 * nb + k] += fabs(dw12);
      n[k] += 1;
    }
  }
}

static void corr_task(void* vctx, int64_t slot) {
  corr_ctx* c = (corr_ctx*)vctx;
  const int nb = c->np * c->nt;
  double* h = c->out + (size_t)slot * ORC_NQ * nb;
  uint64_t* n = c->cnt + (size_t)slot * nb;
  if (c->mode == ORC_GPU_FORMULA) {
    for (int64_t it = c->slot_item_start[slot]; it < c->slot_item_start[slot + 1]; ++it)
      corr_pair(c, c->f1[it], c->f2[it], h, n);
    return;
  }
  /* the CPU backend sums each forest pair into fresh histograms and then adds
   * them to the pixel's (correlation_procedures_cpu.py:40-42, :58-59) */
  double* tmp = (double*)malloc(sizeof(double) * ORC_NQ * (size_t)nb);
  uint64_t* tn = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nb);
  if (!tmp || !tn) { free(tmp); free(tn); return; }
  for (int64_t it = c->slot_item_start[slot]; it < c->slot_item_start[slot + 1]; ++it) {
    memset(tmp, 0, sizeof(double) * ORC_NQ * (size_t)nb);
    memset(tn, 0, sizeof(uint64_t) * (size_t)nb);
    corr_pair(c, c->f1[it], c->f2[it], tmp, tn);
    for (int k = 0; k < ORC_NQ * nb; ++k) h[k] += tmp[k];
    for (int k = 0; k < nb; ++k) n[k] += tn[k];
  }
  free(tmp); free(tn);
}

/* Histograms of the listed forest pairs, accumulated per output slot.  Items
 * [slot_item_start[s], slot_item_start[s+1]) belong to slot s.  out and cnt are
 * accumulated into (not cleared). */
int orc_corr(const orc_forests* F, int64_t nslot, const int64_t* slot_item_start, const int32_t* f1,
             const int32_t* f2, double rpmax, double rtmax, int np, int nt, int mode, int cos_variant,
             double angmax, double* out, uint64_t* cnt, int nthreads) {
  corr_ctx c;
  c.F = F; c.f1 = f1; c.f2 = f2; c.slot_item_start = slot_item_start;
  c.rpmax = rpmax; c.rtmax = rtmax; c.np = np; c.nt = nt; c.mode = mode; c.cos_variant = cos_variant;
  c.angmax = angmax; c.out = out; c.cnt = cnt;
  pool_run(nthreads, nslot, corr_task, &c);
  return 0;
}

/* ------------------------------------------------------------ baseline timing */
/* The reference kernel's own work only (cuda_kernels.cpp:118-159): W and DW of
 * every pixel pair of the listed forest pairs with the FP64 formula of
 * orc_corr (contraction 0), per slot, out[nslot][2][np*nt] accumulated into.
 * Used to time the CPU baseline: no extra outputs, threads over slots. */
typedef struct {
  const orc_forests* F;
  const int32_t *f1, *f2;
  const int64_t* sis;
  double binner_rp, binner_rt;
  int np, nt;
  double* out;
} wdw_ctx;

static void wdw_task(void* vctx, int64_t slot) {
  const wdw_ctx* c = (const wdw_ctx*)vctx;
  const orc_forests* F = c->F;
  const int nb = c->np * c->nt;
  double* hw = c->out + (size_t)slot * 2 * nb;
  double* hd = hw + nb;
  const double fnp = (double)c->np, fnt = (double)c->nt;
  for (int64_t it = c->sis[slot]; it < c->sis[slot + 1]; ++it) {
    const int64_t a = c->f1[it], b = c->f2[it];
    const int64_t s1 = F->start[a], l1 = F->start[a + 1] - s1;
    const int64_t s2 = F->start[b], l2 = F->start[b + 1] - s2;
    const double cos12 = cos12_clamped(F->ux[a], F->uy[a], F->uz[a], F->ux[b], F->uy[b], F->uz[b], 0);
    const double chh = sqrt(0.5 * (1. + cos12)), shh = sqrt(0.5 * (1. - cos12));
    const double* d2 = F->dc + s2;
    const double* w2 = F->w + s2;
    const double* dw2 = F->dw + s2;
    for (int64_t i = 0; i < l1; ++i) {
      const double d1 = F->dc[s1 + i], w1 = F->w[s1 + i], dw1 = F->dw[s1 + i];
      for (int64_t j = 0; j < l2; ++j) {
        const double fp = floor(fabs(d1 - d2[j]) * chh * c->binner_rp);
        const double ft = floor((d1 + d2[j]) * shh * c->binner_rt);
        if (fp >= 0.0 && fp < fnp && ft >= 0.0 && ft < fnt) {
          const int k = (int)fp * c->nt + (int)ft;
          hw[k] += w1 * w2[j];
          hd[k] += dw1 * dw2[j];
        }
      }
    }
  }
}

int orc_corr_wdw(const orc_forests* F, int64_t nslot, const int64_t* slot_item_start, const int32_t* f1,
                 const int32_t* f2, double rpmax, double rtmax, int np, int nt, double* out, int nthreads) {
  wdw_ctx c;
  c.F = F; c.f1 = f1; c.f2 = f2; c.sis = slot_item_start;
  c.binner_rp = (double)np / rpmax; c.binner_rt = (double)nt / rtmax;
  c.np = np; c.nt = nt; c.out = out;
  pool_run(nthreads, nslot, wdw_task, &c);
  return 0;
}

/* ------------------------------------------------------------ adjoint */
typedef struct {
  const orc_forests* F;
  const int32_t* f1;
  const int32_t* f2;
  int64_t nitem;
  double rpmax, rtmax;
  int np, nt, cos_variant;
  const double* coef_dw; /* [nb] g_b / W_b */
  const double* coef_w;  /* [nb] -g_b xi_b / W_b */
  double* g_dw;          /* [npix] */
  double* g_w;           /* [npix] */
} adj_ctx;

/* Gradient of L = sum_b g_b DW_b / W_b with the pair bins held fixed.  The
 * caller supplies coef_dw[b] = g_b / W_b and coef_w[b] = -g_b xi_b / W_b
 * (zero where W_b == 0).  Single-threaded: the scatter touches both forests. */
int orc_adjoint(const orc_forests* F, int64_t nitem, const int32_t* f1, const int32_t* f2, double rpmax,
                double rtmax, int np, int nt, int cos_variant, const double* coef_dw, const double* coef_w,
                double* g_dw, double* g_w) {
  const double binner_rp = (double)np / rpmax, binner_rt = (double)nt / rtmax;
  for (int64_t it = 0; it < nitem; ++it) {
    int64_t a = f1[it], b = f2[it];
    int64_t s1 = F->start[a], l1 = F->start[a + 1] - s1;
    int64_t s2 = F->start[b], l2 = F->start[b + 1] - s2;
    double cos12 = cos12_clamped(F->ux[a], F->uy[a], F->uz[a], F->ux[b], F->uy[b], F->uz[b], cos_variant);
    double chh = sqrt(0.5 * (1. + cos12)), shh = sqrt(0.5 * (1. - cos12));
    for (int64_t i = 0; i < l1; ++i) {
      double d1 = F->dc[s1 + i];
      for (int64_t j = 0; j < l2; ++j) {
        double d2 = F->dc[s2 + j];
        double fp = floor(fabs(d1 - d2) * chh * binner_rp), ft = floor((d1 + d2) * shh * binner_rt);
        if (!(fp >= 0.0 && fp < (double)np && ft >= 0.0 && ft < (double)nt)) continue;
        int k = (int)fp * nt + (int)ft;
        g_dw[s1 + i] += coef_dw[k] * F->dw[s2 + j];
        g_dw[s2 + j] += coef_dw[k] * F->dw[s1 + i];
        g_w[s1 + i] += coef_w[k] * F->w[s2 + j];
        g_w[s2 + j] += coef_w[k] * F->w[s1 + i];
      }
    }
  }
  return 0;
}

/* ------------------------------------------------------------ distortion */
/* FP32 cos of the pair angle from FP32 unit vectors, in the contraction
 * variants of orc_cos12 (cuda_kernels.cpp:72 is the same expression in float). */
static float cos12_f32(float x1, float y1, float z1, float x2, float y2, float z2, int variant) {
  switch (variant) {
    case 0: return fmaf(z1, z2, fmaf(x1, x2, y1 * y2));
    case 1: return fmaf(z1, z2, fmaf(y1, y2, x1 * x2));
    default: {
      float a = x1 * x2, b = y1 * y2, c = z1 * z2;
      return (a + b) + c;
    }
  }
}

/* Pair geometry of one forest pair under a binning mode. */
typedef struct {
  int mode;
  double chh, shh, brp, brt;     /* FP64 binning */
  float ch32, sh32, brp32, brt32; /* FP32 binning */
  int np, nt;
} dist_geom;

static void dist_geom_init(dist_geom* g, const orc_forests* F, int64_t a, int64_t b, double rpmax, double rtmax,
                           int np, int nt, int cos_variant, int mode) {
  g->mode = mode; g->np = np; g->nt = nt;
  if (mode == ORC_BIN_FP32) {
    float c = cos12_f32((float)F->ux[a], (float)F->uy[a], (float)F->uz[a], (float)F->ux[b], (float)F->uy[b],
                        (float)F->uz[b], cos_variant);
    /* cuda_kernels.cpp:73-74: the double literals 0.5 and 1. make the argument
     * an FP64 value, rounded to FP32 by the sqrtf call */
    g->ch32 = sqrtf((float)(0.5 * (1. + (double)c)));
    g->sh32 = sqrtf((float)(0.5 * (1. - (double)c)));
    /* distortion_procedures_pycuda.py:167: float32(numpix / rmax) */
    g->brp32 = (float)((double)np / rpmax);
    g->brt32 = (float)((double)nt / rtmax);
  } else {
    double cos12 = cos12_clamped(F->ux[a], F->uy[a], F->uz[a], F->ux[b], F->uy[b], F->uz[b], cos_variant);
    g->chh = sqrt(0.5 * (1. + cos12));
    g->shh = sqrt(0.5 * (1. - cos12));
    g->brp = (double)np / rpmax;
    g->brt = (double)nt / rtmax;
  }
}

/* (bin_rp, bin_rt) of pixel pair (d1, d2); returns the flat bin or -1. */
static int dist_bin(const dist_geom* g, double d1, double d2, int* bp_out, int* bt_out) {
  if (g->mode == ORC_BIN_FP32) {
    float f1 = (float)d1, f2 = (float)d2;
    float rp = fabsf(f1 - f2) * g->ch32;
    float rt = (f1 + f2) * g->sh32;
    float xp = rp * g->brp32, xt = rt * g->brt32;
    /* int() truncation; NaN and values beyond int range are reported as -1 */
    int bp = (xp == xp && fabsf(xp) < 2.0e9f) ? (int)xp : -1;
    int bt = (xt == xt && fabsf(xt) < 2.0e9f) ? (int)xt : -1;
    if (bp_out) *bp_out = bp;
    if (bt_out) *bt_out = bt;
    if (bp < 0 || bt < 0 || bp >= g->np || bt >= g->nt) return -1;
    return bp * g->nt + bt;
  }
  double fp = floor(fabs(d1 - d2) * g->chh * g->brp), ft = floor((d1 + d2) * g->shh * g->brt);
  if (bp_out) *bp_out = (fp == fp && fabs(fp) < 2.0e9) ? (int)fp : -1;
  if (bt_out) *bt_out = (ft == ft && fabs(ft) < 2.0e9) ? (int)ft : -1;
  if (!(fp >= 0.0 && fp < (double)g->np && ft >= 0.0 && ft < (double)g->nt)) return -1;
  return (int)fp * g->nt + (int)ft;
}

/* bin_rp[i*l2 + j], bin_rt[i*l2 + j] of forest pair (a, b). */
int orc_dist_bins(const orc_forests* F, int32_t a, int32_t b, double rpmax, double rtmax, int np, int nt,
                  int cos_variant, int bin_mode, int32_t* bin_rp, int32_t* bin_rt) {
  dist_geom g;
  dist_geom_init(&g, F, a, b, rpmax, rtmax, np, nt, cos_variant, bin_mode);
  int64_t s1 = F->start[a], l1 = F->start[a + 1] - s1;
  int64_t s2 = F->start[b], l2 = F->start[b + 1] - s2;
  for (int64_t i = 0; i < l1; ++i)
    for (int64_t j = 0; j < l2; ++j) {
      int bp, bt;
      dist_bin(&g, F->dc[s1 + i], F->dc[s2 + j], &bp, &bt);
      bin_rp[i * l2 + j] = bp;
      bin_rt[i * l2 + j] = bt;
    }
  return 0;
}

/* Unnormalised distortion numerator D[A][B] and the bin weights W_B of the
 * listed forest pairs: the reference's compute_etas + compute_d per forest
 * pair (cuda_kernels.cpp:165-278) in FP64, pixel bins from the chosen binning.
 * D and WB are accumulated into.  Scratch is sized per forest pair here. */
int orc_distortion_mode(const orc_forests* F, int64_t nitem, const int32_t* f1, const int32_t* f2, double rpmax,
                        double rtmax, int np, int nt, int cos_variant, int bin_mode, double* D, double* WB) {
  const int nb = np * nt;
  int64_t maxlen = 0;
  for (int64_t f = 0; f < F->n; ++f) if (F->start[f + 1] - F->start[f] > maxlen) maxlen = F->start[f + 1] - F->start[f];
  size_t big = (size_t)nb * (size_t)(maxlen > 0 ? maxlen : 1);
  double* e12 = (double*)malloc(sizeof(double) * big);
  double* e21 = (double*)malloc(sizeof(double) * big);
  double* e13 = (double*)malloc(sizeof(double) * big);
  double* e31 = (double*)malloc(sizeof(double) * big);
  double* e22 = (double*)malloc(sizeof(double) * nb);
  double* e23 = (double*)malloc(sizeof(double) * nb);
  double* e32 = (double*)malloc(sizeof(double) * nb);
  double* e33 = (double*)malloc(sizeof(double) * nb);
  unsigned char* act = (unsigned char*)malloc((size_t)nb);
  int* actlist = (int*)malloc(sizeof(int) * nb);
  int* bins = (int*)malloc(sizeof(int) * (size_t)(maxlen > 0 ? maxlen * maxlen : 1));
  if (!e12 || !e21 || !e13 || !e31 || !e22 || !e23 || !e32 || !e33 || !act || !actlist || !bins) {
    free(e12); free(e21); free(e13); free(e31); free(e22); free(e23); free(e32); free(e33);
    free(act); free(actlist); free(bins);
    return -1;
  }
  for (int64_t it = 0; it < nitem; ++it) {
    int64_t a = f1[it], b = f2[it];
    int64_t s1 = F->start[a], l1 = F->start[a + 1] - s1;
    int64_t s2 = F->start[b], l2 = F->start[b + 1] - s2;
    dist_geom g;
    dist_geom_init(&g, F, a, b, rpmax, rtmax, np, nt, cos_variant, bin_mode);
    /* 1/sum(w) and 1/sum(w dl^2); a forest whose dl are all 0 (e.g. one pixel)
     * has no slope to project out, its slope terms are 0 instead of 0/0 */
    double om1 = F->omega[a], om2 = F->omega[b];
    double io21 = F->odl2[a] > 0.0 ? 1.0 / F->odl2[a] : 0.0, io22 = F->odl2[b] > 0.0 ? 1.0 / F->odl2[b] : 0.0;
    memset(e12, 0, sizeof(double) * (size_t)nb * (size_t)l1);
    memset(e13, 0, sizeof(double) * (size_t)nb * (size_t)l1);
    memset(e21, 0, sizeof(double) * (size_t)nb * (size_t)l2);
    memset(e31, 0, sizeof(double) * (size_t)nb * (size_t)l2);
    memset(e22, 0, sizeof(double) * nb); memset(e23, 0, sizeof(double) * nb);
    memset(e32, 0, sizeof(double) * nb); memset(e33, 0, sizeof(double) * nb);
    memset(act, 0, (size_t)nb);
    /* compute_etas */
    for (int64_t i = 0; i < l1; ++i) {
      double d1 = F->dc[s1 + i], wi = F->w[s1 + i], li = F->dl[s1 + i];
      for (int64_t j = 0; j < l2; ++j) {
        int B = dist_bin(&g, d1, F->dc[s2 + j], 0, 0);
        bins[i * l2 + j] = B;
        if (B < 0) continue;
        double wj = F->w[s2 + j], lj = F->dl[s2 + j];
        act[B] = 1;
        e12[(size_t)B * l1 + i] += wj / om2;
        e21[(size_t)B * l2 + j] += wi / om1;
        e13[(size_t)B * l1 + i] += wj * lj * io22;
        e31[(size_t)B * l2 + j] += wi * li * io21;
        e22[B] += wi * wj / (om1 * om2);
        e23[B] += wi * wj * lj * io22 / om1;
        e32[B] += wi * li * wj * io21 / om2;
        e33[B] += wi * li * wj * lj * io21 * io22;
        WB[B] += wi * wj;
      }
    }
    /* order_active (any order: the sum over B is order-free in exact terms) */
    int nact = 0;
    for (int B = 0; B < nb; ++B) if (act[B]) actlist[nact++] = B;
    /* compute_d */
    for (int64_t i = 0; i < l1; ++i) {
      double wi = F->w[s1 + i], li = F->dl[s1 + i];
      for (int64_t j = 0; j < l2; ++j) {
        int A = bins[i * l2 + j];
        if (A < 0) continue;
        double wj = F->w[s2 + j], lj = F->dl[s2 + j];
        double w12 = wi * wj;
        double* row = D + (size_t)A * nb;
        row[A] += w12;
        for (int q = 0; q < nact; ++q) {
          int B = actlist[q];
          row[B] += w12 * (li * lj * e33[B] + li * e32[B] + lj * e23[B] + e22[B] - li * e31[(size_t)B * l2 + j] -
                           lj * e13[(size_t)B * l1 + i] - e21[(size_t)B * l2 + j] - e12[(size_t)B * l1 + i]);
        }
      }
    }
  }
  free(e12); free(e21); free(e13); free(e31); free(e22); free(e23); free(e32); free(e33);
  free(act); free(actlist); free(bins);
  return 0;
}

int orc_distortion(const orc_forests* F, int64_t nitem, const int32_t* f1, const int32_t* f2, double rpmax,
                   double rtmax, int np, int nt, int cos_variant, double* D, double* WB) {
  return orc_distortion_mode(F, nitem, f1, f2, rpmax, rtmax, np, nt, cos_variant, ORC_BIN_FP64, D, WB);
}
