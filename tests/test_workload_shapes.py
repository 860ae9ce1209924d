"""CPU checks that the seeded synthetic workloads have the configured shapes
(the reference measures no public dataset; these graphs stand in for the
benchmark configurations)."""
import numpy as np


def test_sbm_10k_shape(gen):
    """n = 10,000 in 100 blocks of 100, p_in = 0.1, p_out = 0.0006: about 9.9
    intra and 5.94 inter entries per vertex, both directions, no loops."""
    n, s, d, w, t = gen.sbm(10000, 100, 0.1, 0.0006, 1, 1, 0, with_truth=True)
    assert n == 10000 and np.all(np.bincount(t) == 100)
    assert not np.any(s == d) and np.all(w == 1.0)
    intra = np.sum(t[s] == t[d]) / n
    inter = np.sum(t[s] != t[d]) / n
    assert abs(intra - 0.1 * 99) < 0.03 * 9.9
    assert abs(inter - 0.0006 * 9900) < 0.03 * 5.94
    key = s.astype(np.int64) * n + d
    assert np.all(np.diff(key) > 0)                         # sorted, duplicates merged
    assert np.array_equal(np.sort(d.astype(np.int64) * n + s), key)   # symmetric


def test_lfr_shape(gen):
    """n = 2^20, degrees from a power law of exponent 2.5 on [5, 5000],
    community sizes exponent 1.5 on [50, 50000], mixing 0.3, unit weights."""
    n, s, d, w, t = gen.lfr(with_truth=True)
    assert n == 1 << 20 and not np.any(s == d) and np.all(w == 1.0)
    deg = np.bincount(s, minlength=n)
    k = np.arange(5, 5001, dtype=np.float64)
    mean = (k * k ** -2.5).sum() / (k ** -2.5).sum()        # 13.17
    assert abs(deg.mean() - mean) < 0.08 * mean
    assert deg.max() <= 5000 and np.mean(deg < 5) < 0.01   # merged duplicates cost a few vertices an edge
    assert abs(np.mean(t[s] != t[d]) - 0.3) < 0.02
    sizes = np.bincount(t)
    sizes = sizes[sizes > 0]
    assert sizes.min() >= 50 and sizes.max() <= 50000


def test_rmat_shape(gen):
    """R-MAT scale 16, edge factor 16: self loops dropped, duplicates merged
    by summing integer weights, symmetric; the degree skew of (0.57, 0.19,
    0.19, 0.05) puts the heaviest rows at the lowest ids."""
    n, s, d, w = gen.rmat(16)
    assert n == 1 << 16 and not np.any(s == d)
    assert np.all(w == np.round(w)) and w.min() >= 1.0
    key = s.astype(np.int64) * n + d
    assert np.all(np.diff(key) > 0)
    assert np.array_equal(np.sort(d.astype(np.int64) * n + s), key)
    # at most 16 * 2^16 generated edges, both directions after symmetrising
    assert len(s) <= 2 * 16 * n
    deg = np.bincount(s, minlength=n)
    assert deg[: n // 16].sum() > deg[-(n // 16):].sum() * 20
