"""Host-side logic: catalogue packing, slots, sharding, healpix, synthetic data."""
import numpy as np
import pytest

from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import owner_slots
from lya2pcf_b200.forests import from_quasar_dict
from lya2pcf_b200.healpix import ang2pix_ring, radec_to_pix
from lya2pcf_b200.sharding import shard_slots, slot_costs


def test_healpix_ring_basics():
    # every pixel of a fine sphere sampling is hit exactly in [0, 12 nside^2)
    for nside in (1, 2, 4, 16):
        th = np.arccos(np.linspace(-0.9999, 0.9999, 300))
        ph = np.linspace(0, 2 * np.pi, 301)[:-1]
        T, Ph = np.meshgrid(th, ph)
        p = ang2pix_ring(nside, T.ravel(), Ph.ravel())
        assert p.min() == 0 and p.max() == 12 * nside * nside - 1
        assert len(np.unique(p)) == 12 * nside * nside
    # ring ordering: north cap pixels first, pixel index grows towards the south
    assert ang2pix_ring(16, 0.01, 0.3) < ang2pix_ring(16, np.pi / 2, 0.3) < ang2pix_ring(16, np.pi - 0.01, 0.3)
    # equator, phi = 0 at nside 1 is pixel 4
    assert ang2pix_ring(1, np.pi / 2, 0.0) == 4
    # equal-area: a uniform sphere sample fills the 192 pixels of nside 4 evenly
    rng = np.random.default_rng(0)
    z = rng.uniform(-1, 1, 400000); phi = rng.uniform(0, 2 * np.pi, 400000)
    counts = np.bincount(ang2pix_ring(4, np.arccos(z), phi), minlength=192)
    assert counts.std() / counts.mean() < 0.03


def test_owner_slots_contiguous():
    slot, pix = owner_slots([7, 7, 3, 3, 3, 9])
    assert slot.tolist() == [0, 0, 1, 1, 1, 2] and pix.tolist() == [7, 3, 9]
    with pytest.raises(ValueError):
        owner_slots([1, 2, 1])


def test_shard_slots_balanced():
    """LPT shares partition the slots; their loads differ by at most the
    largest slot cost."""
    rng = np.random.default_rng(1)
    costs = rng.uniform(0, 10, 1000)
    for world in (1, 2, 3, 8):
        sh = shard_slots(costs, world)
        assert len(sh) == world
        assert np.array_equal(np.sort(np.concatenate(sh)), np.arange(len(costs)))
        tot = [costs[s].sum() for s in sh]
        assert max(tot) - min(tot) <= costs.max() + 1e-9


def test_slot_costs():
    c = slot_costs([2, 3, 4], [0, 0, 1], [1, 2, 2], [0, 1, 1], 2)
    assert c.tolist() == [2 * 3 + 2 * 4, 3 * 4]


def test_synthetic_shapes_and_determinism():
    a = synthetic.make(0)
    b = synthetic.make(0)
    assert a.n == 2000 and np.array_equal(a.dc, b.dc) and np.array_equal(a.pix, b.pix)
    L = a.lengths
    assert L.min() >= 150 and L.max() <= 600
    assert np.all(np.diff(a.pix) >= 0)            # grouped by healpix pixel
    c1 = synthetic.make(1, scale=0.01)
    assert c1.lengths.max() <= 614 and c1.lengths.min() >= 50
    for f in range(0, c1.n, 97):                  # dc sorted inside every forest
        d = c1.forest(f)['dc']
        assert np.all(np.diff(d) > 0)
    # same-quasar twins exist and share the name
    _, cnt = np.unique(c1.name, return_counts=True)
    assert (cnt == 2).sum() >= 1
    # healpix pixel of each forest
    assert np.array_equal(c1.pix, radec_to_pix(16, c1.ra, c1.dec))


def test_quasar_dict_round_trip():
    fs = synthetic.make(4, n=40)
    data = fs.to_quasar_dict()
    fs2, forests = from_quasar_dict(data)
    assert fs2.n == fs.n
    assert np.array_equal(fs2.dc, fs.dc) and np.array_equal(fs2.w, fs.w) and np.array_equal(fs2.dw, fs.dw)
    np.testing.assert_allclose(fs2.z, fs.z, rtol=1e-12)
    assert forests[0].__class__.__module__ == 'forest_class'
