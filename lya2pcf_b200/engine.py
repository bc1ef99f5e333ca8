"""Host-side driver of the native pair-binning library.

:class:`PairEngine` owns one library context on one GPU: it uploads a
:class:`~lya2pcf_b200.forests.ForestSet`, builds (or receives) the forest-pair
work queue, runs the histogram kernels and copies results back.  It is the
layer under the drop-in ``correlation_procedures_pycuda`` module and the
benchmark.
"""
import ctypes as C

import numpy as np

from . import _native as N
from . import parameters as P


def owner_slots(pix):
    """Slot index of every forest: pixels numbered in order of first appearance.

    Forests of one pixel must be contiguous (as in a pixel dict).  Returns
    ``(slot_of_forest int32, slot_pixels int64)``."""
    pix = np.asarray(pix, dtype=np.int64)
    if pix.size == 0:
        return np.zeros(0, dtype=np.int32), np.zeros(0, dtype=np.int64)
    change = np.ones(pix.size, dtype=bool)
    change[1:] = pix[1:] != pix[:-1]
    slot = (np.cumsum(change) - 1).astype(np.int32)
    slot_pixels = pix[change]
    if len(np.unique(slot_pixels)) != len(slot_pixels):
        raise ValueError('forests of one healpix pixel must be contiguous in forest order')
    return slot, slot_pixels


class PairEngine:
    """One GPU context of the pair-binning library."""

    def __init__(self, device=0, rpmax=P.rpmax, rtmax=P.rtmax, np_=P.numpix_rp, nt=P.numpix_rt):
        self.lib = N.load()
        self.ctx = C.c_void_p()
        N.check(self.lib.lya_ctx_create(int(device), C.byref(self.ctx)))
        self.np_, self.nt = int(np_), int(nt)
        self.nb = self.np_ * self.nt
        self.rpmax, self.rtmax = float(rpmax), float(rtmax)
        self._check(self.lib.lya_set_bins(self.ctx, self.rpmax, self.rtmax, self.np_, self.nt))
        self.fs = None
        self.slot_pixels = None
        self.n_pairs = 0
        self._keep = []
        self.tuned = {}   # kernel -> {'variant', 'run_cap'} chosen by autotune

    def _check(self, rc):
        N.check(rc, self.ctx)

    def close(self):
        if self.ctx:
            self.lib.lya_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ upload
    def upload(self, fs):
        slot, slot_pixels = owner_slots(fs.pix)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        arrs = dict(start=np.ascontiguousarray(fs.start, dtype=np.int64), dc=f64(fs.dc), w=f64(fs.w),
                    dw=f64(fs.dw), z=f64(fs.z), dl=f64(fs.dl), ux=f64(fs.ux), uy=f64(fs.uy), uz=f64(fs.uz),
                    ra=f64(fs.ra), dec=f64(fs.dec), name=np.ascontiguousarray(fs.name, dtype=np.int64),
                    slot=np.ascontiguousarray(slot, dtype=np.int32), omega=f64(fs.omega), odl2=f64(fs.odl2))
        p = N.ptr
        self._check(self.lib.lya_upload_forests(
            self.ctx, fs.n, p(arrs['start']), p(arrs['dc']), p(arrs['w']), p(arrs['dw']), p(arrs['z']),
            p(arrs['dl']), p(arrs['ux']), p(arrs['uy']), p(arrs['uz']), p(arrs['ra']), p(arrs['dec']),
            p(arrs['name']), p(arrs['slot']), int(len(slot_pixels)), p(arrs['omega']), p(arrs['odl2'])))
        self.fs = fs
        self.slot_of_forest = slot
        self.slot_pixels = slot_pixels
        self.n_pairs = 0
        return self

    def upload_deltas(self, fs, delta, loglam, project=True):
        """Upload the geometry and weights of ``fs`` with per-pixel ``delta`` and
        log10(lambda) ``loglam``; the projection of ``quasar.fill_dw``
        (``forest_class.py:48-68``) runs on the device.  ``fs.dw``, ``fs.dl``,
        ``fs.omega`` and ``fs.odl2`` are not read; :meth:`projection` returns
        the device's."""
        slot, slot_pixels = owner_slots(fs.pix)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        arrs = dict(start=np.ascontiguousarray(fs.start, dtype=np.int64), dc=f64(fs.dc), w=f64(fs.w),
                    delta=f64(delta), z=f64(fs.z), loglam=f64(loglam), ux=f64(fs.ux), uy=f64(fs.uy), uz=f64(fs.uz),
                    ra=f64(fs.ra), dec=f64(fs.dec), name=np.ascontiguousarray(fs.name, dtype=np.int64),
                    slot=np.ascontiguousarray(slot, dtype=np.int32))
        p = N.ptr
        self._check(self.lib.lya_upload_deltas(
            self.ctx, fs.n, p(arrs['start']), p(arrs['dc']), p(arrs['w']), p(arrs['delta']), p(arrs['z']),
            p(arrs['loglam']), p(arrs['ux']), p(arrs['uy']), p(arrs['uz']), p(arrs['ra']), p(arrs['dec']),
            p(arrs['name']), p(arrs['slot']), int(len(slot_pixels)), 1 if project else 0))
        self.fs = fs
        self.slot_of_forest = slot
        self.slot_pixels = slot_pixels
        self.n_pairs = 0
        return self

    def projection(self):
        """``(dw[npix], dl[npix], omega[n], odl2[n])`` of the uploaded catalogue."""
        n, npix = self.fs.n, self.fs.npix_total
        dw, dl, om, o2 = np.zeros(npix), np.zeros(npix), np.zeros(n), np.zeros(n)
        self._check(self.lib.lya_get_projection(self.ctx, N.ptr(dw), N.ptr(dl), N.ptr(om), N.ptr(o2)))
        return dw, dl, om, o2

    # ------------------------------------------------------------------ work queue
    def build_pairs(self, angmax):
        """Neighbour search on the device (``quasar.neighborhood`` for every forest)."""
        n = C.c_int64(0)
        self._check(self.lib.lya_build_pairs(self.ctx, float(angmax), float(np.cos(angmax)), C.byref(n)))
        self.n_pairs = int(n.value)
        return self.n_pairs

    def set_pairs(self, f1, f2):
        f1 = np.ascontiguousarray(f1, dtype=np.int32)
        f2 = np.ascontiguousarray(f2, dtype=np.int32)
        if f1.shape != f2.shape:
            raise ValueError('f1 and f2 differ in length')
        self._check(self.lib.lya_set_pairs(self.ctx, len(f1), N.ptr(f1), N.ptr(f2)))
        self.n_pairs = len(f1)

    def select_slots(self, slots):
        """Keep only the work-queue pairs whose first forest's owner slot is in
        ``slots`` (an iterable of slot indices, or a boolean mask over the
        slots): the rank-local queue of a sharded run.  Returns the pairs kept."""
        n = len(self.slot_pixels)
        keep = np.zeros(n, dtype=np.uint8)
        slots = np.asarray(slots)
        if slots.dtype == bool:
            if slots.shape != (n,):
                raise ValueError(f'slot mask must have {n} entries')
            keep[slots] = 1
        else:
            keep[slots.astype(np.int64)] = 1
        self._check(self.lib.lya_select_slots(self.ctx, N.ptr(keep)))
        self.n_pairs = int(self.stats()['n_pairs'])
        return self.n_pairs

    def get_pairs(self):
        f1 = np.zeros(max(self.n_pairs, 1), dtype=np.int32)
        f2 = np.zeros(max(self.n_pairs, 1), dtype=np.int32)
        self._check(self.lib.lya_get_pairs(self.ctx, N.ptr(f1), N.ptr(f2)))
        return f1[:self.n_pairs], f2[:self.n_pairs]

    # ------------------------------------------------------------------ correlation
    def run(self, kernel=N.KERNEL_FP32_GUARDED, guard=1e-4, warps=0, blocks_per_sm=0, slots=None, variant=None,
            run_cap=None):
        """Histograms of the work queue (restricted to owner slots
        ``range(*slots)`` when given).  ``variant`` and ``run_cap`` default to
        the library's defaults, or to the choice of :meth:`autotune` for this
        kernel when it ran.  Returns :meth:`stats`."""
        s0, s1 = (0, 0) if slots is None else (int(slots[0]), int(slots[1]))
        tuned = self.tuned.get(int(kernel), {})
        variant = tuned.get('variant', 0) if variant is None else variant
        run_cap = tuned.get('run_cap', 0) if run_cap is None else run_cap
        opts = N.CorrOpts(int(kernel), float(guard), int(warps), int(blocks_per_sm), s0, s1, int(variant),
                          int(run_cap))
        self._check(self.lib.lya_corr_run(self.ctx, C.byref(opts)))
        return self.stats()

    def autotune(self, kernel=N.KERNEL_FP32_GUARDED, guard=1e-4, fraction=0.05, variants=None, run_caps=(64, 128, 256),
                 seed=0):
        """Choose the diagonal walk and the run-length cap of ``kernel`` for this
        catalogue: time every candidate on a contiguous range of owner slots
        holding about ``fraction`` of the work queue's pixel pairs (the second
        of two runs, so each candidate is timed from its captured graph) and
        keep the fastest for later :meth:`run` calls.  Walks: 0 (the FP32
        kernel's lean walk, two diagonals per lane otherwise), 2 (two
        diagonals per lane) and 1 (one per lane).  Returns the timings."""
        if variants is None:
            variants = (0, 2, 1) if int(kernel) == N.KERNEL_FP32_GUARDED else (0, 2)
        slots = self._sample_slots(fraction, seed)
        timings = []
        for v in variants:
            for cap in run_caps:
                for _ in range(2):
                    st = self.run(kernel=kernel, guard=guard, slots=slots, variant=v, run_cap=cap)
                timings.append({'variant': v, 'run_cap': cap, 'kernel_ms': st['kernel_ms']})
        best = min(timings, key=lambda r: r['kernel_ms'])
        self.tuned[int(kernel)] = {'variant': best['variant'], 'run_cap': best['run_cap']}
        return {'best': dict(self.tuned[int(kernel)]), 'slots': list(slots), 'timings': timings}

    def _sample_slots(self, fraction, seed):
        """A contiguous owner-slot range with about ``fraction`` of the queue's
        reference pixel pairs, starting at a seeded random slot."""
        f1, f2 = self.get_pairs()
        L = self.fs.lengths.astype(np.float64)
        per_slot = np.bincount(self.slot_of_forest[f1], weights=L[f1] * L[f2], minlength=len(self.slot_pixels))
        total = per_slot.sum()
        start = int(np.random.default_rng(seed).integers(0, max(1, len(per_slot))))
        acc, end = 0.0, start
        while end < len(per_slot) and acc < fraction * total:
            acc += per_slot[end]
            end += 1
        while start > 0 and acc < fraction * total:   # reached the last slot: extend downwards
            start -= 1
            acc += per_slot[start]
        return (start, max(end, start + 1))

    def timer_start(self):
        """Record a start event on the library's stream."""
        self._check(self.lib.lya_timer(self.ctx, 0, None))

    def timer_stop(self):
        """Record a stop event, wait for it; device milliseconds since timer_start."""
        ms = C.c_double(0.0)
        self._check(self.lib.lya_timer(self.ctx, 1, C.byref(ms)))
        return ms.value

    def sync(self):
        self._check(self.lib.lya_sync(self.ctx))

    def histograms(self, slot_first=0, n=None, out=None, counts_out=None):
        """``(hist[n, 5, nb] float64, counts[n, nb] uint64)`` for slots
        ``slot_first .. slot_first+n-1`` (W, DW, RP, RT, Z sums; see _native.Q_*)."""
        nslots = len(self.slot_pixels)
        n = nslots - slot_first if n is None else int(n)
        hist = out if out is not None else np.zeros((n, N.NQ, self.nb), dtype=np.float64)
        cnt = counts_out if counts_out is not None else np.zeros((n, self.nb), dtype=np.uint64)
        self._check(self.lib.lya_corr_get(self.ctx, int(slot_first), n, N.ptr(hist), N.ptr(cnt)))
        return hist, cnt

    def adjoint(self, g, out_dw=None, out_w=None):
        """Gradient of sum_b g_b DW_b/W_b w.r.t. dw and w of every pixel (CSR
        order), bins held fixed.  ``g`` is a numpy array or a CUDA float64
        torch tensor on this context's device.  ``out_dw``/``out_w`` may be
        CUDA torch tensors (float64, contiguous, on this context's device) to
        receive the result on the device; otherwise numpy arrays are returned."""
        flags = 0
        if hasattr(g, 'data_ptr'):
            if g.numel() != self.nb:
                raise ValueError(f'g must have {self.nb} entries')
            gp = C.c_void_p(g.data_ptr())
            flags |= 2
        else:
            g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1)
            if g.size != self.nb:
                raise ValueError(f'g must have {self.nb} entries')
            gp = N.ptr(g)
        if out_dw is not None:
            self._check(self.lib.lya_corr_adjoint(self.ctx, gp, C.c_void_p(out_dw.data_ptr()),
                                                  C.c_void_p(out_w.data_ptr()), flags | 1))
            return out_dw, out_w
        gdw = np.zeros(self.fs.npix_total, dtype=np.float64)
        gw = np.zeros(self.fs.npix_total, dtype=np.float64)
        self._check(self.lib.lya_corr_adjoint(self.ctx, gp, N.ptr(gdw), N.ptr(gw), flags))
        return gdw, gw

    def totals(self, out_w=None, out_dw=None):
        """``(W[nb], DW[nb])``: sum w1w2 and sum dw1dw2 over every owner slot of
        the last :meth:`run`.  With CUDA float64 torch tensors ``out_w`` and
        ``out_dw`` (on this context's device) the totals stay on the device."""
        if out_w is not None:
            self._check(self.lib.lya_corr_totals(self.ctx, C.c_void_p(out_w.data_ptr()),
                                                 C.c_void_p(out_dw.data_ptr()), 1))
            return out_w, out_dw
        W = np.zeros(self.nb)
        DW = np.zeros(self.nb)
        self._check(self.lib.lya_corr_totals(self.ctx, N.ptr(W), N.ptr(DW), 0))
        return W, DW

    def update_weights(self, w, dw):
        """Replace w and dw of every pixel (numpy arrays, or CUDA float64 torch
        tensors on this context's device)."""
        if hasattr(w, 'data_ptr'):
            self._check(self.lib.lya_update_weights(self.ctx, C.c_void_p(w.data_ptr()), C.c_void_p(dw.data_ptr()), 1))
        else:
            w = np.ascontiguousarray(w, dtype=np.float64)
            dw = np.ascontiguousarray(dw, dtype=np.float64)
            self._check(self.lib.lya_update_weights(self.ctx, N.ptr(w), N.ptr(dw), 0))

    def distortion(self):
        """Distortion numerator D[nb, nb] and bin weights W[nb] over the work
        queue (FP64).  The normalised matrix of ``distortion.py`` is D / W[:, None]."""
        D = np.zeros((self.nb, self.nb), dtype=np.float64)
        W = np.zeros(self.nb, dtype=np.float64)
        self._check(self.lib.lya_dist_run(self.ctx, N.ptr(D), N.ptr(W)))
        return D, W

    DIST_SHAPES = ((512, 32), (512, 16), (512, 24), (256, 32), (256, 16))   # lya_dist_config shapes

    def autotune_distortion(self, fraction=0.05, min_items=2000):
        """Choose the distortion kernel's launch shape (threads per CTA, pixels
        per staged chunk) for this catalogue: time every shape on the first
        ``fraction`` of the work queue (at least ``min_items`` forest pairs;
        the second of two runs, i.e. the replayed graph) and keep the fastest
        for later :meth:`distortion` calls.  Shapes whose shared memory does not
        fit the catalogue's longest forest are skipped.  Returns the timings."""
        n = max(min_items, int(self.n_pairs * fraction))
        timings = []
        for shape in range(len(self.DIST_SHAPES)):
            self._check(self.lib.lya_dist_config(self.ctx, shape, n))
            try:
                for _ in range(2):
                    self._check(self.lib.lya_dist_run(self.ctx, None, None))
            except N.LyaError as err:
                timings.append({'shape': shape, 'error': str(err)})
                continue
            timings.append({'shape': shape, 'threads': self.DIST_SHAPES[shape][0],
                            'chunk': self.DIST_SHAPES[shape][1], 'kernel_ms': self.stats()['kernel_ms']})
        ok = [t for t in timings if 'kernel_ms' in t]
        best = min(ok, key=lambda t: t['kernel_ms'])['shape'] if ok else 0
        self._check(self.lib.lya_dist_config(self.ctx, best, 0))
        return {'best': best, 'items': n, 'timings': timings}

    def covariance(self, smooth=True):
        """Covariance of the per-owner-slot correlation estimates xi = DW/W of
        the last :meth:`run`, computed on the device from its histograms (the
        reading loop and ``cov``/``cov_smooth`` of ``post_processing.py``).
        Returns ``(mean[nb], cov[nb, nb], cov_smooth[nb, nb] or None, smoothed)``."""
        mean = np.zeros(self.nb)
        c = np.zeros((self.nb, self.nb))
        self._check(self.lib.lya_covariance(self.ctx, 0, None, None, N.ptr(mean), N.ptr(c)))
        if not smooth:
            return mean, c, None, False
        cs = np.zeros_like(c)
        sm = C.c_int32(0)
        self._check(self.lib.lya_covariance_smooth(self.ctx, None, N.ptr(cs), C.byref(sm)))
        return mean, c, cs, bool(sm.value)

    def stats(self):
        st = N.Stats()
        self._check(self.lib.lya_stats(self.ctx, C.byref(st)))
        return st.as_dict()
