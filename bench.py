"""Benchmark of the lya2pcf pair-binning path on B200.

Metric: pixel pairs binned per second.  A pixel pair is one pair (i in f1,
j in f2) of a neighbouring forest pair as the reference enumerates them
(``forest_class.quasar.neighborhood``), i.e. the unit of work of the
reference's ``pair_correlation`` kernel; a step counts sum(len1 * len2) over
its forest pairs whether or not the kernel needed to evaluate every pair.

One step = the whole job on one catalogue resident in HBM: device neighbour
search (work queue) + the per-slot histograms (W, DW, counts, RP, RT, Z) in
one persistent launch.  Workload: the 150,000-forest synthetic catalogue
(8,000 deg^2, 50x50 bins to 200 Mpc/h).  With N GPUs every rank bins its own
catalogue of that size (different seed): weak scaling, no data-path
collective.  ``--split`` instead shares one catalogue among the N ranks as
the drop-in drivers do: every rank holds the whole catalogue and neighbour
queue, keeps the pairs of its LPT share of the owner pixels
(``lya_select_slots``) and bins them (strong scaling, no data-path
collective); its step is neighbour search + share selection + histograms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --profile-case corr|dist|adjoint [--config C] [--scale S]

``--profile-case`` runs one pass of one hot kernel on a catalogue of the
given configuration and scale (after one warm-up pass) and prints the
library's statistics: the command line the ncu captures under ``profiles/``
profile, on cases whose inputs exceed L2 while holding a few GB at most.

Prints one JSON line (rank 0).  Its ``roofline`` is the pair kernel's FP32
issue bound (the kernel is neither HBM- nor tensor-bound); the HBM figure and
the shared-atomic term sit inside it as sub-objects.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'pixel-pairs binned/s: FP32-guarded vs plain FP64 GPU at bit-exact counts'
UNIT = 'pixel-pairs/s'
WORKLOAD = ('150,000 synthetic Lyman-alpha forests on 8,000 deg^2 (19/deg^2), lengths U[50,700] clamped to the '
            '614-pixel log-lambda grid, 50x50 (r_par, r_perp) bins to 200 Mpc/h, float64 inputs')
GUARD = 1e-4     # Mpc/h guard band of the FP32 kernel
DMMA_PEAK_TFLOPS = 40.0   # B200 FP64 tensor-core rate, data sheet (the distortion's block products)
KERNEL_CODES = {'fp32': 0, 'fp64diag': 1, 'fp64plain': 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--config', type=int, default=1)
    ap.add_argument('--scale', type=float, default=1.0)
    ap.add_argument('--kernel', default='fp32', choices=list(KERNEL_CODES))
    ap.add_argument('--split', action='store_true',
                    help='share one catalogue among the ranks by owner pixel (strong scaling)')
    ap.add_argument('--e2e-steps', type=int, default=2)
    ap.add_argument('--cpu-seconds', type=float, default=15.0, help='target CPU-baseline sample duration')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-compare', action='store_true', help='skip the FP64 comparison sample')
    ap.add_argument('--no-full-compare', action='store_true',
                    help='skip the whole-catalogue FP64 runs of the comparison (about a minute)')
    ap.add_argument('--no-ref-kernel', action='store_true',
                    help="skip timing the reference's own CUDA kernel (oracle/_ref) on the comparison sample")
    ap.add_argument('--no-autotune', action='store_true', help='library default walk instead of the autotuned one')
    ap.add_argument('--dist-scale', type=float, default=0.03,
                    help='distortion sample: fraction of the 30,000-forest distortion catalogue (0 = skip)')
    ap.add_argument('--no-adjoint', action='store_true', help='skip the adjoint timing')
    ap.add_argument('--no-covariance', action='store_true', help='skip the covariance post-processing timing')
    ap.add_argument('--profile-case', choices=['corr', 'dist', 'adjoint'], default=None,
                    help='one pass of one hot kernel (after a warm-up pass), for profilers')
    ap.add_argument('--variant', type=int, default=0, help='--profile-case corr: walk variant')
    return ap.parse_args()


# ---------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self, want):
        self.world = int(os.environ.get('WORLD_SIZE', '1'))
        self.rank = int(os.environ.get('RANK', '0'))
        self.local = int(os.environ.get('LOCAL_RANK', '0'))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            backend = 'nccl' if self._cuda() else 'gloo'
            if backend == 'nccl':
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    @staticmethod
    def _cuda():
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        dev = torch.device('cuda', self.local) if self._cuda() else torch.device('cpu')
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if not self.pg:
            return v
        import torch
        dev = torch.device('cuda', self.local) if self._cuda() else torch.device('cpu')
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(suffix='.csv')
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(gpu_index),
                 '--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
                 'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
                 'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap',
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(',')]
                if len(parts) >= 8:
                    rows.append(parts)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace('.', '', 1).isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace('.', '', 1).isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[k] for r in rows for k in range(4) if 'Active' in r[4 + k] and 'Not' not in r[4 + k]})
        busy = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)]
        return {'sm_mhz': statistics.median(busy or sm) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(rows)}


# ---------------------------------------------------------------- CPU baseline (oracle port)
def cpu_baseline(fs, angmax, seconds, seed=5):
    """Time the CPU restatement of the reference kernel (the oracle's W/DW-only
    path, orc_corr_wdw: the work pair_correlation does, at the single-thread
    rate of the reference's numba kernel) on a bounded, seeded sample of the
    same catalogue's work, all host cores: forest pairs
    (the reference's per-launch unit) in a seeded random order, in batches of
    one chunk of about 1e8 pixel pairs per core, until the elapsed time
    reaches ``seconds``."""
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0))
    off, nbr = O.neighbours(fs, angmax, nthreads=cores)
    f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
    L = fs.lengths.astype(np.float64)
    order = np.random.default_rng(seed).permutation(len(f1))
    cost = L[f1[order]] * L[f2[order]]
    csum = np.cumsum(cost)
    done, pairs, dt, calls = 0, 0.0, 0.0, 0
    while done < len(order) and dt < seconds:
        # the next `cores` chunks of ~1e8 pixel pairs each, one per thread
        base = csum[done - 1] if done else 0.0
        bounds = np.searchsorted(csum, base + 1e8 * np.arange(1, cores + 1), side='right')
        bounds = np.minimum(np.maximum(bounds, done + 1), len(order))
        cuts = np.unique(np.concatenate([[done], bounds]))
        idx = order[cuts[0]:cuts[-1]]
        sis_c = (cuts - cuts[0]).astype(np.int64)
        t = time.perf_counter()
        O.corr_wdw(fs, f1[idx], f2[idx], sis_c, nthreads=cores)
        dt += time.perf_counter() - t
        pairs += float(np.sum(cost[cuts[0]:cuts[-1]]))
        done = int(cuts[-1])
        calls += 1
    return {'value': pairs / dt, 'unit': UNIT, 'cores': cores, 'kind': 'port',
            'sample': f'{done} of {len(f1)} forest pairs (seeded random order, {calls} calls of {cores} chunks of '
                      f'~1e8 pixel pairs), {pairs:.3e} pixel pairs, {dt:.1f} s; FP64 W and DW of every pixel pair, '
                      f'the reference kernel\'s work (single-thread rate 1.08x the reference numba kernel\'s, '
                      f'oracle/time_numba_vs_port.py)',
            'seconds': dt, 'pairs': pairs}


def build_catalog(config, scale, rank):
    """The catalogue of ``rank``: its own seed (weak scaling), or rank 0's for
    every rank when ``rank`` is 0 (the shared catalogue of ``--split``)."""
    from lya2pcf_b200 import synthetic
    seed = synthetic.SEEDS[config] + 1000 * rank
    fs = synthetic.make(config, scale=scale, seed=seed)
    return fs, synthetic.angmax_for(fs)


# ---------------------------------------------------------------- reference arm
def run_reference(args, dist):
    fs, angmax = build_catalog(args.config, args.scale, 0)
    vals = []
    base = None
    for k in range(args.warmup + args.steps):
        b = cpu_baseline(fs, angmax, args.cpu_seconds / 2 if k < args.warmup else args.cpu_seconds, seed=5 + k)
        if k >= args.warmup:
            vals.append(b['value'])
            base = b
    value = float(np.median(vals))
    return {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': int(os.environ.get('WORLD_SIZE', args.gpus)),
            'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * base['seconds'], 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'impl': 'reference',
            'config': {'workload': WORKLOAD, 'forests': fs.n, 'config': args.config, 'scale': args.scale},
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': base['cores'], 'kind': base['kind'],
                             'sample': base['sample']},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


# ---------------------------------------------------------------- B200 arm
def pinned_copy(a):
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


def run_b200(args, dist):
    import torch
    from lya2pcf_b200 import _native as N
    from lya2pcf_b200.engine import PairEngine, owner_slots

    dev = dist.local
    torch.cuda.set_device(dev)
    fs, angmax = build_catalog(args.config, args.scale, 0 if args.split else dist.rank)
    kern = KERNEL_CODES[args.kernel]
    eng = PairEngine(device=dev).upload(fs)
    share = None
    if args.split:
        from lya2pcf_b200.sharding import shard_slots, slot_costs
        eng.build_pairs(angmax)
        f1, f2 = eng.get_pairs()
        costs = slot_costs(fs.lengths, f1, f2, eng.slot_of_forest, len(eng.slot_pixels))
        share = shard_slots(costs, dist.world)[dist.rank]
        share_frac = float(costs[share].sum() / max(costs.sum(), 1.0))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        pass

    def step():
        eng.build_pairs(angmax)
        if share is not None:
            eng.select_slots(share)
        return eng.run(kernel=kern, guard=GUARD)

    tune = None
    for k in range(args.warmup):
        if k == 1 and not args.no_autotune:   # after the first warm-up step: choose the walk, then warm it
            tune = eng.autotune(kernel=kern, guard=GUARD)
        step()
    st0 = eng.stats()
    launches0 = st0['launches']
    dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev) if dist.rank == 0 else None
    kernel_ms, build_ms, run_ms = [], [], []
    eng.timer_start()
    for _ in range(args.steps):
        st = step()
        kernel_ms.append(st['kernel_ms'])
        build_ms.append(st['build_ms'])
        run_ms.append(st['run_ms'])
    dev_ms = eng.timer_stop()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop() if clocks else None
    st = eng.stats()
    launches = st['launches'] - launches0
    ref_pairs = st['ref_pairs']
    t_max = dist.max(dev_ms)
    pairs_all = dist.sum(ref_pairs * args.steps)
    value = pairs_all / (t_max * 1e-3)

    # ---- e2e through the C ABI with host buffers (pinned), copies inside the region
    slot, slot_pixels = owner_slots(fs.pix)
    host = {}
    keep = []
    for k, a in dict(start=fs.start.astype(np.int64), dc=fs.dc, w=fs.w, dw=fs.dw, z=fs.z, dl=fs.dl, ux=fs.ux,
                     uy=fs.uy, uz=fs.uz, ra=fs.ra, dec=fs.dec, name=fs.name.astype(np.int64),
                     slot=slot.astype(np.int32), omega=fs.omega, odl2=fs.odl2).items():
        host[k], t = pinned_copy(np.ascontiguousarray(a))
        keep.append(t)
    nslot = len(slot_pixels)
    hist_out, t1 = pinned_copy(np.zeros((nslot, N.NQ, eng.nb), dtype=np.float64))
    cnt_out, t2 = pinned_copy(np.zeros((nslot, eng.nb), dtype=np.uint64))
    keep += [t1, t2]
    h2d = int(sum(a.nbytes for a in host.values()))
    d2h = int(hist_out.nbytes + cnt_out.nbytes)
    L = N.load()
    p = N.ptr

    def e2e_step():
        N.check(L.lya_upload_forests(eng.ctx, fs.n, p(host['start']), p(host['dc']), p(host['w']), p(host['dw']),
                                     p(host['z']), p(host['dl']), p(host['ux']), p(host['uy']), p(host['uz']),
                                     p(host['ra']), p(host['dec']), p(host['name']), p(host['slot']), nslot,
                                     p(host['omega']), p(host['odl2'])), eng.ctx)
        eng.build_pairs(angmax)
        if share is not None:
            eng.select_slots(share)
        eng.run(kernel=kern, guard=GUARD)
        N.check(L.lya_corr_get(eng.ctx, 0, nslot, p(hist_out), p(cnt_out)), eng.ctx)

    e2e_value = None
    e2e_phases = None
    if args.e2e_steps > 0:
        e2e_step()
        dist.barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = dist.max(time.perf_counter() - t)
        e2e_value = dist.sum(ref_pairs * args.e2e_steps) / e2e_s
        e2e_phases = e2e_itemised(eng, e2e_step_parts(L, eng, fs, host, nslot, hist_out, cnt_out, angmax, kern,
                                                      share))
        e2e_phases['wall_ms_per_step'] = 1e3 * e2e_s / args.e2e_steps

    # ---- covariance of the per-owner-pixel correlations of the last run (post-processing, on the device)
    covariance = None
    if not args.no_covariance:
        try:
            t = time.perf_counter()
            eng.covariance()
            first_s = time.perf_counter() - t
            t = time.perf_counter()
            mean, cmat, csm, smoothed = eng.covariance()
            cov_s = time.perf_counter() - t
            covariance = {'seconds': cov_s, 'first_call_seconds': first_s,
                          'gram_kernels_ms': eng.stats()['kernel_ms'], 'rows': len(slot_pixels),
                          'bins': eng.nb, 'smoothed': smoothed,
                          'gram_fma': float(len(slot_pixels)) * eng.nb * eng.nb,
                          'what': 'lya_covariance (rows from the run on the device, FP64 tensor-core Gram) + '
                                  'lya_covariance_smooth, wall clock with the 50 MB copies out (second call; '
                                  'the first, with its host and device allocations, in first_call_seconds)'}
        except N.LyaError as err:
            covariance = {'error': str(err)}

    # ---- adjoint (gradient of sum_b g_b DW_b/W_b w.r.t. dw and w of every pixel) on the same catalogue
    adjoint = None
    if not args.no_adjoint:
        g = np.random.default_rng(4).normal(size=eng.nb)
        gdw = torch.empty(fs.npix_total, dtype=torch.float64, device=f'cuda:{dev}')
        gw = torch.empty_like(gdw)
        eng.adjoint(g, out_dw=gdw, out_w=gw)
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.adjoint(g, out_dw=gdw, out_w=gw)
        torch.cuda.synchronize()
        adj_s = time.perf_counter() - t
        adjoint = {'seconds': adj_s, 'ref_pixel_pairs_per_s': ref_pairs / adj_s,
                   'what': 'one lya_corr_adjoint call (device gradients) over the whole work queue, wall clock',
                   'forward_kernel_ms': float(np.median(kernel_ms))}

    out = None
    if dist.rank == 0:
        # ---- FP32 vs FP64 on a sample of owner slots: bit-exact counts and pairs/s
        compare = None
        if not args.no_compare:
            compare = fp64_comparison(eng, fs, kern, full=not args.no_full_compare,
                                      ref_kernel=not args.no_ref_kernel)
        # ---- roofline of the dominant kernel (the pair kernel): FP32 issue bound
        kms = float(np.median(kernel_ms))
        roof = alu_roofline(st, kms, clk)
        algo_bytes = st['ref_pixels'] * 24.0          # dc, w, dw (FP64) of both forests per forest pair
        achieved_gbs = algo_bytes / (kms * 1e-3) / 1e9
        hbm = peaks.get('hbm_gbs')
        roof['traffic'] = dram_traffic_per_launch(st['ref_pairs'])
        roof['kernel'] = 'k_corr<FP32_GUARDED> (pair kernel, lean walk)'
        roof['kernel_ms'] = kms
        roof['hbm'] = {'bound': 'hbm', 'achieved': achieved_gbs, 'peak': hbm if hbm else 6650.0, 'unit': 'GB/s',
                       'frac': achieved_gbs / (hbm if hbm else 6650.0),
                       'peak_source': 'measured (MEASURED_PEAKS.json)' if hbm else 'fallback',
                       'algorithmic_bytes_per_launch': algo_bytes,
                       'note': 'not the bound: per forest pair the kernel reads (len1+len2) x 24 B algorithmically, '
                               're-read from L2'}
        roof['smem_atomic'] = smem_atomic_term(st, kms, dev)
        cpu = None if args.no_cpu_baseline else cpu_baseline(fs, angmax, args.cpu_seconds)
        distortion = None if args.dist_scale <= 0 else distortion_sample(args.dist_scale, dev)
        ms_step = t_max / args.steps
        out = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': dist.world, 'steps': args.steps,
               'warmup': args.warmup, 'ms_per_step': ms_step, 'higher_is_better': True,
               'scaling': 'strong' if args.split else 'weak',
               'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (seeded catalogue, no public data set)',
               'config': {'workload': WORKLOAD, 'config': args.config, 'scale': args.scale, 'forests': fs.n,
                          'owner_pixels': nslot, 'forest_pairs': st['n_pairs'],
                          'ref_pixel_pairs_per_step': ref_pairs, 'kernel': args.kernel, 'guard_mpc_h': GUARD,
                          'guard_bound_mpc_h': st['guard_bound'], 'l2': 'inputs larger than L2 '
                          f'({fs.npix_total * 52 / 1e9:.1f} GB resident catalogue)',
                          'step': 'device neighbour search + histogram run',
                          'parallelism': (f'split: {dist.world} rank(s) share one catalogue by owner pixel (LPT on '
                                          f'the pair count; rank 0 holds {share_frac:.3f} of it)') if args.split
                          else f'weak: {dist.world} rank(s), one catalogue each'},
               'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                       'path': 'lya_upload_forests + lya_build_pairs + lya_corr_run + lya_corr_get, pinned host',
                       'phases': e2e_phases},
               'tuned': tune, 'kernel_ms_steps': kernel_ms, 'run_ms_steps': run_ms, 'build_ms_steps': build_ms,
               'distortion': distortion, 'adjoint': adjoint, 'covariance': covariance,
               'gpu_launches': int(launches),
               'kernel_ms': kms, 'build_ms': float(np.median(build_ms)),
               'evaluated_pairs_per_step': st['evaluated_pairs'], 'guard_rechecks_per_step': st['guard_rechecks'],
               'guard_fraction': st['guard_rechecks'] / max(st['evaluated_pairs'], 1.0),
               'roofline': roof, 'clocks': clk, 'cpu_baseline': cpu, 'fp64_comparison': compare}
    eng.close()
    return out


def e2e_step_parts(L, eng, fs, host, nslot, hist_out, cnt_out, angmax, kern, share=None):
    """The four C-ABI calls of one end-to-end step, as separate callables."""
    from lya2pcf_b200 import _native as N
    p = N.ptr
    return [
        ('upload', lambda: N.check(L.lya_upload_forests(
            eng.ctx, fs.n, p(host['start']), p(host['dc']), p(host['w']), p(host['dw']), p(host['z']), p(host['dl']),
            p(host['ux']), p(host['uy']), p(host['uz']), p(host['ra']), p(host['dec']), p(host['name']),
            p(host['slot']), nslot, p(host['omega']), p(host['odl2'])), eng.ctx)),
        ('build_pairs', lambda: (eng.build_pairs(angmax), eng.select_slots(share) if share is not None else None)),
        ('run', lambda: eng.run(kernel=kern, guard=GUARD)),
        ('get', lambda: N.check(L.lya_corr_get(eng.ctx, 0, nslot, p(hist_out), p(cnt_out)), eng.ctx)),
    ]


def e2e_itemised(eng, parts):
    """One more end-to-end step with each call bracketed by device events on
    the library's stream (timer_start / timer_stop) and the host clock: where
    an end-to-end step's time goes."""
    out = {}
    for name, fn in parts:
        eng.sync()
        t = time.perf_counter()
        eng.timer_start()
        fn()
        dev_ms = eng.timer_stop()
        out[name] = {'device_ms': dev_ms, 'wall_ms': 1e3 * (time.perf_counter() - t)}
    out['sum_wall_ms'] = sum(v['wall_ms'] for v in out.values())
    st = eng.stats()
    out['run_kernel_ms'] = st['kernel_ms']
    out['build_kernels_ms'] = st['build_ms']
    return out


def distortion_sample(scale, dev):
    """Distortion matrix (all neighbouring forest pairs, no subsampling) of a
    seeded sample of the 30,000-forest log-normal distortion catalogue:
    ``scale`` of its forests on the same sky density."""
    from lya2pcf_b200 import synthetic
    from lya2pcf_b200.engine import PairEngine
    fs = synthetic.make(3, scale=scale)
    am = synthetic.angmax_for(fs)
    with PairEngine(device=dev) as eng:
        eng.upload(fs)
        n = eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        L = fs.lengths.astype(np.float64)
        ref = float(np.sum(L[f1] * L[f2]))
        tune = eng.autotune_distortion()
        eng.distortion()
        D, W = eng.distortion()
        st = eng.stats()
        ms = st['kernel_ms']
    flops = st['dist_mma_flops']
    return {'forests': fs.n, 'scale': scale, 'forest_pairs': n, 'ref_pixel_pairs': ref, 'kernel_ms': ms,
            'forest_pairs_per_s': n / (ms * 1e-3), 'ref_pixel_pairs_per_s': ref / (ms * 1e-3),
            'matrix': f'{D.shape[0]}x{D.shape[1]} float64, {int(np.count_nonzero(D))} nonzero',
            'tuned': tune,
            'roofline': {'bound': 'fp64_tensor', 'achieved': flops / (ms * 1e-3) / 1e12, 'unit': 'TFLOP/s',
                         'peak': DMMA_PEAK_TFLOPS, 'frac': flops / (ms * 1e-3) / 1e12 / DMMA_PEAK_TFLOPS,
                         'flops': flops,
                         'peak_source': 'nominal B200 FP64 tensor-core rate (data sheet, not measured)',
                         'what': 'flops of the column block products (8x8 tiles over the staged rows, counted '
                                 'by the kernel; run as m16n8k8 FP64 MMAs)'}}


XI_FLOOR_FRAC = 0.1   # per-bin xi errors are stated over bins with |xi| >= this fraction of the median |xi|


def xi_errors(h32, h64):
    """Error of xi = DW/W of the FP32-guarded histograms against the FP64
    kernel's (which equals the oracle to 1e-12 in the tests), per owner pixel
    and bin: normwise (max |dxi| / max |xi|) and per bin (|dxi| / |xi|) over the
    bins whose |xi| is at least XI_FLOOR_FRAC of the median nonzero |xi|."""
    W32, W64 = h32[:, 0], h64[:, 0]
    xi32 = np.divide(h32[:, 1], W32, out=np.zeros_like(W32), where=W32 != 0)
    xi64 = np.divide(h64[:, 1], W64, out=np.zeros_like(W64), where=W64 != 0)
    d = np.abs(xi32 - xi64)
    a = np.abs(xi64)
    nz = a > 0
    floor = XI_FLOOR_FRAC * float(np.median(a[nz])) if nz.any() else 0.0
    sel = a >= floor if nz.any() else nz
    rel = d[sel] / a[sel] if sel.any() else np.zeros(1)
    return {'normwise_max_dxi_over_max_xi': float(d.max() / max(a.max(), 1e-300)),
            'per_bin_floor_xi': floor, 'per_bin_floor_rule': f'|xi| >= {XI_FLOOR_FRAC} x median nonzero |xi|',
            'per_bin_bins': int(sel.sum()), 'per_bin_max_rel_err': float(rel.max()),
            'per_bin_median_rel_err': float(np.median(rel)),
            'per_bin_fraction_within_1e-6': float(np.mean(rel <= 1e-6))}


def fp64_comparison(eng, fs, kern, full=True, ref_kernel=True):
    """FP32-guarded vs the FP64 kernels: a 40-owner-pixel sample (accuracy,
    counts, pairs/s, and the reference's own CUDA kernel on the same pixels
    when oracle/_ref was built), then the whole catalogue once per kernel
    (counts equal in every bin of every pixel, and the speed-ups)."""
    from lya2pcf_b200.engine import owner_slots
    slot, pixels = owner_slots(fs.pix)
    nslot = len(pixels)
    rng = np.random.default_rng(9)
    s0 = int(rng.integers(0, max(1, nslot - 40)))
    rngs = (s0, min(nslot, s0 + 40))
    res = {}
    counts = {}
    hists = {}
    for name, code in (('fp32_guarded', 0), ('fp64_diagonal', 1), ('fp64_plain', 2)):
        st = eng.run(kernel=code, guard=GUARD, slots=rngs)
        st = eng.run(kernel=code, guard=GUARD, slots=rngs)
        h, c = eng.histograms(rngs[0], rngs[1] - rngs[0])
        counts[name] = c
        hists[name] = h
        res[name] = {'pairs_per_s': st['run_ref_pairs'] / (st['kernel_ms'] * 1e-3), 'kernel_ms': st['kernel_ms'],
                     'W_sum': float(h[:, 0].sum())}
    res['slots'] = list(rngs)
    res['ref_pairs'] = st['run_ref_pairs']
    res['counts_equal_fp32_fp64diag'] = bool(np.array_equal(counts['fp32_guarded'], counts['fp64_diagonal']))
    res['counts_equal_fp32_fp64plain'] = bool(np.array_equal(counts['fp32_guarded'], counts['fp64_plain']))
    # accuracy of the FP32-guarded sums against the FP64 kernel (equal to the oracle to 1e-12 in the tests)
    h32, h64 = hists['fp32_guarded'], hists['fp64_plain']
    W32, W64 = h32[:, 0], h64[:, 0]
    nz = W64 > 0
    res['max_rel_err_W'] = float(np.max(np.abs(W32 - W64)[nz] / W64[nz])) if nz.any() else 0.0
    res['max_rel_err_RP_RT_Z'] = [float(np.max(np.abs(h32[:, q] - h64[:, q])[nz] / np.abs(h64[:, q])[nz]))
                                  for q in (2, 3, 4)] if nz.any() else None
    res['xi'] = xi_errors(h32, h64)
    res['speedup_fp32_vs_fp64plain'] = res['fp32_guarded']['pairs_per_s'] / res['fp64_plain']['pairs_per_s']
    res['speedup_fp32_vs_fp64diag'] = res['fp32_guarded']['pairs_per_s'] / res['fp64_diagonal']['pairs_per_s']
    if ref_kernel:
        res['reference_kernel'] = reference_kernel_sample(eng, fs, rngs, counts['fp64_plain'])
        rk = res['reference_kernel']
        if rk and rk.get('pairs_per_s'):
            res['speedup_fp32_vs_reference_kernel'] = res['fp32_guarded']['pairs_per_s'] / rk['pairs_per_s']
    if full:
        res['whole_catalogue'] = whole_catalogue_comparison(eng)
    return res


def whole_catalogue_comparison(eng):
    """Every owner pixel of the catalogue with each kernel once: pixel pairs
    per second from the kernel events, and pair counts of the FP64 kernels
    equal to the FP32-guarded kernel's in every bin of every pixel."""
    out = {}
    c32 = None
    for name, code in (('fp32_guarded', 0), ('fp64_diagonal', 1), ('fp64_plain', 2)):
        st = eng.run(kernel=code, guard=GUARD)
        _, c = eng.histograms()
        out[name] = {'kernel_ms': st['kernel_ms'], 'pairs_per_s': st['run_ref_pairs'] / (st['kernel_ms'] * 1e-3),
                     'evaluated_pairs': st['evaluated_pairs']}
        if c32 is None:
            c32 = c
        else:
            out[f'counts_equal_fp32_{name}'] = bool(np.array_equal(c32, c))
    out['ref_pairs'] = st['run_ref_pairs']
    out['speedup_fp32_vs_fp64plain'] = out['fp32_guarded']['pairs_per_s'] / out['fp64_plain']['pairs_per_s']
    out['speedup_fp32_vs_fp64diag'] = out['fp32_guarded']['pairs_per_s'] / out['fp64_diagonal']['pairs_per_s']
    return out


def reference_kernel_sample(eng, fs, rngs, counts64):
    """The reference's own pair_correlation (cuda_kernels.cpp:90-162, compiled
    from the reference tree into oracle/_ref) on the same owner pixels, driven
    per first forest as two_point_per_pixel does
    (correlation_procedures_pycuda.py:141-166): a baseline, not the product.
    Its W must have as many nonzero bins as the FP64 kernel's counts."""
    from oracle import ref as R
    if not R.available():
        return {'unavailable': 'oracle/_ref/libref_kernels.so was not built (needs the reference tree at build time)'}
    f1, f2 = eng.get_pairs()
    sel = (eng.slot_of_forest[f1] >= rngs[0]) & (eng.slot_of_forest[f1] < rngs[1])
    f1, f2 = f1[sel], f2[sel]
    firsts, starts = np.unique(f1, return_index=True)
    ends = np.append(starts[1:], len(f1))
    lists = [f2[a:b] for a, b in zip(starts, ends)]
    L = fs.lengths.astype(np.float64)
    ref_pairs = float(np.sum(L[f1] * L[f2]))
    ms, w_hist, _ = R.corr_timed(fs, firsts, lists)
    return {'pairs_per_s': ref_pairs / (ms * 1e-3), 'loop_ms': ms, 'ref_pairs': ref_pairs, 'launches': len(firsts),
            'nonzero_bins_match': bool(np.array_equal(w_hist.ravel() != 0, counts64.sum(0) != 0)),
            'what': 'reference pair_correlation, one launch + synchronize per first forest, FP64 global atomics'}


def dram_traffic_per_launch(ref_pairs):
    """DRAM bytes per pair-kernel launch from the committed ncu capture
    (profiles/k_corr_fp32.json), scaled to this launch's pixel pairs."""
    try:
        prof = json.load(open(os.path.join(ROOT, 'profiles', 'k_corr_fp32.json')))
        return prof['dram_bytes'] / prof['ref_pairs'] * ref_pairs
    except Exception:
        return None


def alu_roofline(st, kms, clk):
    """The pair kernel against its FP32 issue bound: evaluated pixel pairs per
    second against the B200's FP32 lane rate divided by the FP32 operations one
    pixel pair needs (10 in the reference kernel, cuda_kernels.cpp:142-155: rp
    sub+mul, rt add+mul, two bin scalings, two weight products, two
    accumulations; 7 more for the new outputs: three products and four
    accumulations).  The lane rate is 148 SMs x 128 FP32 lanes x the SM clock
    sampled during the timed steps (computed, not measured)."""
    evals = st['evaluated_pairs'] / (kms * 1e-3)
    sm_mhz = (clk or {}).get('sm_mhz') or 1965.0
    fp32_lanes = 148 * 128 * sm_mhz * 1e6        # FP32 lane-instructions per second
    ops = 17.0
    bound = fp32_lanes / ops
    return {'bound': 'fp32_issue', 'achieved': evals, 'peak': bound, 'unit': 'pair-evaluations/s',
            'frac': evals / bound, 'fp32_ops_per_pair': ops, 'sm_mhz_used': sm_mhz,
            'peak_source': 'computed: 148 SMs x 128 FP32 lanes x sampled SM clock / 17 ops per pair (not measured)'}


def smem_atomic_term(st, kms, dev):
    """The shared-memory atomic term of the bound: the reference algorithm does
    6 shared atomics (5 FP64 sums and a count) per in-range pixel pair; the
    kernel does 6 per run of pairs that share a bin.  Peak atomic rate measured
    here by the library's probe (lya_probe_smem_atomics, FP64 adds into random
    bins of a 2500-bin histogram)."""
    from lya2pcf_b200 import _native as N
    rates = np.zeros(3)
    N.check(N.load().lya_probe_smem_atomics(int(dev), N.ptr(rates)))
    rate = float(rates[1])
    evals = max(st['evaluated_pairs'], 1.0)
    f_in = st['in_range_pairs'] / evals
    per_pair_ref = 6.0 * f_in
    per_pair_kernel = 6.0 * st['runs_flushed'] / evals
    return {'peak_atomics_per_s': rate, 'probe_rates_per_s': {'f64_distinct': float(rates[0]),
                                                              'f64_random_bins': rate,
                                                              'u32_distinct': float(rates[2])},
            'source': 'measured in this run: lya_probe_smem_atomics, FP64 shared atomicAdd into random bins',
            'in_range_fraction': f_in,
            'bound_pair_evals_per_s_reference_form': rate / per_pair_ref if per_pair_ref else None,
            'atomics_per_evaluated_pair': per_pair_kernel,
            'bound_pair_evals_per_s_this_kernel': rate / per_pair_kernel if per_pair_kernel else None,
            'atomic_time_fraction': (st['runs_flushed'] * 6.0 / rate) / (kms * 1e-3)}


def profile_case(args):
    """One pass of the pair kernel, the distortion kernel or the adjoint on a
    catalogue of configuration ``args.config`` at ``args.scale``, after one
    warm-up pass; prints the library's statistics as one JSON line."""
    from lya2pcf_b200 import synthetic
    from lya2pcf_b200.engine import PairEngine
    fs = synthetic.make(args.config, scale=args.scale)
    kern = KERNEL_CODES[args.kernel]
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(synthetic.angmax_for(fs))
        if args.profile_case == 'dist':
            tune = eng.autotune_distortion()
            eng.distortion()
            t = time.perf_counter()
            eng.distortion()
            st = eng.stats()
            st['dist_wall_s'] = time.perf_counter() - t
            st['tuned'] = tune
            st['forest_pairs'] = eng.n_pairs
        elif args.profile_case == 'adjoint':
            eng.run(kernel=kern, guard=GUARD)
            g = np.random.default_rng(4).normal(size=eng.nb)
            eng.adjoint(g)
            t = time.perf_counter()
            eng.adjoint(g)
            st = eng.stats()
            st['adjoint_wall_s'] = time.perf_counter() - t
        else:
            eng.run(kernel=kern, guard=GUARD, variant=args.variant)
            st = eng.run(kernel=kern, guard=GUARD, variant=args.variant)
        st['npix_total'] = fs.npix_total
        st['case'] = {'kernel': args.profile_case, 'config': args.config, 'scale': args.scale, 'forests': fs.n}
        print(json.dumps(st), flush=True)


def main():
    args = parse()
    if args.split:   # the extras below describe one catalogue on one GPU; a split run measures the step only
        args.no_compare = args.no_adjoint = args.no_covariance = True
        args.dist_scale = 0.0
    if args.profile_case:
        profile_case(args)
        return
    if args.impl == 'reference':
        # the reference path is CPU code: rank 0 alone runs it, other ranks exit
        if int(os.environ.get('RANK', '0')) != 0:
            return
        out = run_reference(args, None)
        print(json.dumps(out), flush=True)
        return
    dist = Dist(args.gpus)
    try:
        out = run_b200(args, dist)
        if dist.rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


if __name__ == '__main__':
    main()
