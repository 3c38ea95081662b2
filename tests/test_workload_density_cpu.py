"""The synthetic density fields of the benchmark boxes
(platoanalyze_b200/workloads.py): the smoothed field against an independent
restatement of its recipe (seeded U[0,1] noise, separable Gaussian with
sigma cells truncated at 3 sigma, half-sample-symmetric borders, affine
rescale to [0,1], clip), its x-fastest layout and the per-tet repetition."""
import numpy as np

from platoanalyze_b200.workloads import cell_density, hex_density


def fold(i, n):
    """Index of a half-sample-symmetric extension (d c b a | a b c d | d c b a)."""
    i = i % (2 * n)
    return i if i < n else 2 * n - 1 - i


def smooth_axis(a, axis, sigma):
    r = int(3.0 * sigma + 0.5)
    w = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    w /= w.sum()
    a = np.moveaxis(a, axis, -1)
    n = a.shape[-1]
    out = np.zeros_like(a)
    for i in range(n):
        for k, wk in zip(range(-r, r + 1), w):
            out[..., i] += wk * a[..., fold(i + k, n)]
    return np.moveaxis(out, -1, axis)


def recipe(dims, seed, sigma, lo, hi):
    nx, ny, nz = dims
    f = np.random.default_rng(seed).uniform(0.0, 1.0, (nz, ny, nx))
    for axis in range(3):
        f = smooth_axis(f, axis, sigma)
    f = (f - f.min()) / (f.max() - f.min())
    return np.clip(f, lo, hi).ravel()


def test_smoothed_field_follows_its_recipe():
    # axes shorter than the filter radius (9 cells at sigma = 3) exercise repeated folding
    for dims, sigma in (((12, 10, 8), 3.0), ((7, 5, 4), 1.5)):
        got = hex_density(dims, 1234, kind="smoothed", sigma=sigma, lo=0.01, hi=1.0)
        want = recipe(dims, 1234, sigma, 0.01, 1.0)
        assert np.allclose(got, want, rtol=0, atol=1e-12)
        assert got.min() == 0.01 and got.max() == 1.0


def test_layout_seed_and_per_tet_repetition():
    dims = (6, 5, 4)
    h = hex_density(dims, 7)
    assert np.array_equal(h, hex_density(dims, 7))
    assert not np.array_equal(h, hex_density(dims, 8))
    c = cell_density(dims, 7)
    assert c.shape == (6 * 6 * 5 * 4,)
    assert np.array_equal(c.reshape(-1, 6), np.repeat(h[:, None], 6, axis=1))
    # x fastest: hex (i, j, k) sits at i + nx (j + ny k)
    grid = h.reshape(4, 5, 6)
    assert grid[2, 3, 1] == h[1 + 6 * (3 + 5 * 2)]
    u = hex_density(dims, 3, kind="uniform", lo=0.3, hi=1.0)
    assert u.min() >= 0.3 and u.max() < 1.0
