"""Failure paths on the GPU, made on the host (no GPU fault is caused).

* A device error flag: lya_debug_inject makes the next run's pair kernel raise
  its error flag (the flag the kernel sets when it finds a run record outside
  the histogram); the run returns LYA_ERR_DEVICE, and the next run on the same
  context gives the oracle's histograms.
* Allocation failures: lya_debug_fail_alloc makes one device allocation of the
  library fail; the call that made it returns LYA_ERR_ALLOC, and calling it
  again on the same context succeeds, with results equal to the oracle."""
import numpy as np
import pytest

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def small():
    fs = synthetic.make(0, scale=0.05)
    am = synthetic.angmax_for(fs)
    off, nbr = O.neighbours(fs, am)
    f1, f2, sis, _ = O.items_from_csr(fs, off, nbr)
    _, co = O.corr(fs, f1, f2, sis)
    return fs, am, co


def test_device_error_flag_reaches_the_caller(small):
    fs, am, co = small
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        N.check(eng.lib.lya_debug_inject(eng.ctx, 1), eng.ctx)
        with pytest.raises(N.LyaError) as ei:
            eng.run(kernel=N.KERNEL_FP32_GUARDED)
        assert ei.value.code == 7 and 'error flag' in str(ei.value)
        with pytest.raises(N.LyaError):            # no result after a failed run
            eng.histograms()
        eng.run(kernel=N.KERNEL_FP32_GUARDED)      # the context is still usable
        _, c = eng.histograms()
        assert np.array_equal(c, co)


@pytest.mark.parametrize('after', [0, 3, 12, 25, 31])
def test_one_failed_allocation_then_recovery(small, after):
    """Fail the allocation made after `after` more allocations: wherever it
    falls (context, upload, neighbour search, run), exactly one call fails
    with LYA_ERR_ALLOC, a second attempt of that call succeeds, and the
    histograms equal the oracle's."""
    fs, am, co = small
    lib = N.load()
    failures = []
    eng = None
    lib.lya_debug_fail_alloc(after)
    try:
        steps = [('create', lambda: PairEngine()), ('upload', lambda: eng.upload(fs)),
                 ('build', lambda: eng.build_pairs(am)), ('run', lambda: eng.run(kernel=N.KERNEL_FP32_GUARDED)),
                 ('get', lambda: eng.histograms())]
        out = None
        for name, fn in steps:
            try:
                r = fn()
            except N.LyaError as err:
                assert err.code == 3, (name, err)
                failures.append(name)
                r = fn()
            if name == 'create':
                eng = r
            out = r
        assert len(failures) <= 1
        _, c = out
        assert np.array_equal(c, co)
    finally:
        lib.lya_debug_fail_alloc(-1)
        if eng is not None:
            eng.close()
    if after <= 3:
        assert failures, 'an early allocation must have failed'
