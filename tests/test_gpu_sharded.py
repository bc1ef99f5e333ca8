"""Owner-pixel shares on the GPU: the drop-in module's restrict_pixels path.

Ranks of the drivers share no data path for the correlation: every rank
uploads the whole catalogue, builds the whole neighbour queue, keeps the pairs
of its LPT share of the owner pixels (lya_select_slots) and bins only those.
Here the ranks of a 2- and a 3-rank split run one after the other in one
process on one GPU (they never wait on one another), and the union of their
pixels is checked against the CPU oracle: every pixel exactly once, counts
bit-exact, sums within the FP32 kernel's tolerance (1e-6 relative; DW against
sum |dw1 dw2|)."""
import numpy as np
import pytest

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.dropin_path import ensure_on_path
from lya2pcf_b200.engine import PairEngine
from lya2pcf_b200.sharding import shard_slots, slot_costs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('world', [2, 3])
def test_dropin_shares_cover_every_pixel_once(world):
    ensure_on_path()
    import correlation_procedures_pycuda as cp
    fs = synthetic.make(0, scale=0.2)
    data = fs.to_quasar_dict()
    am = synthetic.angmax_for(fs)
    cp.init(data, None, (50, 50), am)
    eng = cp._engine
    f1, f2 = eng.get_pairs()
    costs = slot_costs(eng.fs.lengths, f1, f2, eng.slot_of_forest, len(eng.slot_pixels))
    pixels = [int(p) for p in eng.slot_pixels]
    seen = {}
    for rank, share in enumerate(shard_slots(costs, world)):
        mine = [pixels[s] for s in share]
        cp.restrict_pixels(mine)
        for p in pixels:
            w, dw = cp.two_point_per_pixel(p)
            c = cp.pixel_extras(p)['npairs']
            if p in mine:
                assert p not in seen
                seen[p] = (w.ravel(), dw.ravel(), c.ravel())
            else:
                assert not w.any() and not c.any()
    assert sorted(seen) == sorted(pixels)
    off, nbr = O.neighbours(eng.fs, am)
    of1, of2, sis, opix = O.items_from_csr(eng.fs, off, nbr)
    ho, co = O.corr(eng.fs, of1, of2, sis)
    for s, p in enumerate(opix.tolist()):
        w, dw, c = seen[int(p)]
        assert np.array_equal(c, co[s]), p
        assert np.all(np.abs(w - ho[s, O.Q_W]) <= 1e-6 * ho[s, O.Q_W])
        assert np.all(np.abs(dw - ho[s, O.Q_DW]) <= 1e-6 * ho[s, O.Q_DWABS] + 1e-300)


def test_select_slots_keeps_only_the_share():
    fs = synthetic.make(0, scale=0.1)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        share = np.arange(1, len(eng.slot_pixels), 2)
        assert len(share) >= 2
        kept = eng.select_slots(share)
        g1, g2 = eng.get_pairs()
        sel = np.isin(eng.slot_of_forest[f1], share)
        assert kept == int(sel.sum()) > 0
        assert np.array_equal(g1, f1[sel]) and np.array_equal(g2, f2[sel])
        L = fs.lengths
        assert eng.stats()['ref_pairs'] == float(np.sum(L[g1] * L[g2]))
        eng.run(kernel=N.KERNEL_FP32_GUARDED)
        _, c = eng.histograms()
        outside = np.setdiff1d(np.arange(len(eng.slot_pixels)), share)
        assert c[outside].sum() == 0 and c[share].sum() > 0
        assert eng.select_slots(np.zeros(len(eng.slot_pixels), dtype=bool)) == 0
