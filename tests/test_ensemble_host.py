"""Host side of the uneven ensembles: the pooled layout helpers, the member
generator and the argument checks the library makes before touching a GPU."""
import numpy as np
import pytest

from scale_b200 import hevi, mkinit


def test_pool_unpool_round_trip():
    rng = np.random.default_rng(0)
    shapes = [(6, 5, 4), (3, 7, 2), (4, 4, 4)]
    n3 = [int(np.prod(s)) for s in shapes]
    off = np.concatenate([[0], np.cumsum(n3)])
    for ncomp in (1, 3):
        arrs = [np.asfortranarray(rng.standard_normal(s + ((ncomp,) if ncomp > 1 else ()))) for s in shapes]
        pooled = hevi.pool(arrs, off, ncomp=ncomp)
        assert pooled.size == ncomp * off[-1]
        # component q of member m sits at q*total + offset[m]
        for m, a in enumerate(arrs):
            q = ncomp - 1
            comp = a[..., q] if ncomp > 1 else a
            got = pooled[q * off[-1] + off[m]: q * off[-1] + off[m] + n3[m]]
            assert np.array_equal(got, np.ravel(comp, order="F"))
        back = hevi.unpool(pooled, off, shapes, ncomp=ncomp)
        for a, b in zip(arrs, back):
            assert np.array_equal(a, b)


def test_pool_vectors_with_slots():
    KA = [6, 4]
    off = np.array([0, 6, 10])
    fdz = [np.arange(1.0, 6.0), np.arange(10.0, 13.0)]  # KA-1 values each
    p = hevi.pool(fdz, off, slots=KA)
    assert p.tolist() == [1, 2, 3, 4, 5, 0, 10, 11, 12, 0]
    with pytest.raises(ValueError):
        hevi.pool([np.zeros(7), np.zeros(3)], off, slots=KA)


def test_ensemble_members():
    cs = mkinit.ensemble(scale=1 / 16)
    assert len(cs) == 48
    sizes = sorted({(c.g.IMAX, c.g.JMAX, c.g.KMAX) for c in cs})
    assert sizes == [(8, 8, 64), (8, 8, 96), (16, 16, 96)]
    full = [(I, J, K) for (I, J, K) in mkinit.ENSEMBLE_SIZES]
    assert full.count((64, 64, 64)) == full.count((128, 128, 96)) == full.count((256, 256, 96)) == 16
    # each member has its own bubble and noise
    a, b = mkinit.ensemble(sizes=[(16, 16, 20)] * 2)
    assert not np.array_equal(a.state["RHOT"], b.state["RHOT"])
    assert a.dt == b.dt and a.nd_coef == b.nd_coef


def test_ensemble_setup_argument_checks():
    idx = mkinit.ensemble(sizes=[(16, 12, 20)])[0].g.index_dict()
    with pytest.raises(hevi.HeviError, match="members"):
        hevi.ensemble_setup([idx] * 65)
    with pytest.raises(hevi.HeviError, match="members"):
        hevi.ensemble_setup([])
    bad = dict(idx, KE=idx["KE"] + 1)
    with pytest.raises(hevi.HeviError, match="inconsistent"):
        hevi.ensemble_setup([idx, bad])


def test_bubble_on_its_support_equals_full_domain_sum():
    """The input generator adds each warm bubble only where it is nonzero; the
    state equals the full-domain formula bit for bit."""
    rng = np.random.default_rng(3)
    for g in (mkinit.uniform_grid(40, 40, 80, 500.0, 500.0, 250.0),
              mkinit.stretched_grid(24, 20, 30, 250.0, 250.0, 50.0, 400.0)):
        base = mkinit.base_state(g)
        full = mkinit._bcast(base["pott"], g)
        part = full.copy(order="F")
        Lx, Ly = g.IMAX * g.DX, g.JMAX * g.DY
        for _ in range(6):
            b = (rng.uniform(0, Lx), rng.uniform(0, Ly), rng.uniform(500, 4000), rng.uniform(1e3, 6e3),
                 rng.uniform(1e3, 6e3), rng.uniform(1e3, 4e3), rng.uniform(1, 4))
            full = full + b[6] * mkinit.bubble(g, *b[:6])
            part = mkinit.add_bubble(part, g, *b)
        assert np.array_equal(full, part)
