"""The SIMP design loop's host pieces (platoanalyze_b200/workloads.py) that
make the 64^3 training and benchmark designs: the sensitivity filter against
a brute-force restatement of its formula, and the optimality-criteria update's
constraints (volume, move limit, bounds) and monotonicity."""
import numpy as np

from platoanalyze_b200.workloads import oc_update, sensitivity_filter


def brute_filter(rho, dc, dims, radius):
    """dc_i = sum_j H_ij rho_j dc_j / (max(rho_i, 1e-3) sum_j H_ij), with
    H_ij = max(0, radius - |x_i - x_j|) over hex centres inside the box."""
    nx, ny, nz = dims
    idx = [(i, j, k) for k in range(nz) for j in range(ny) for i in range(nx)]
    out = np.empty(len(idx))
    for a, (i, j, k) in enumerate(idx):
        num = den = 0.0
        for b, (p, q, r) in enumerate(idx):
            h = max(0.0, radius - np.sqrt((i - p) ** 2 + (j - q) ** 2 + (k - r) ** 2))
            num += h * rho[b] * dc[b]
            den += h
        out[a] = num / (max(rho[a], 1e-3) * den)
    return out


def test_sensitivity_filter_matches_its_formula():
    dims = (5, 4, 3)
    rng = np.random.default_rng(0)
    n = dims[0] * dims[1] * dims[2]
    rho = rng.uniform(1e-4, 1.0, n)  # includes values below the 1e-3 floor
    rho[3] = 1e-5
    dc = -rng.uniform(0.1, 2.0, n)
    for radius in (1.5, 2.2):
        got = sensitivity_filter(rho, dc, dims, radius=radius)
        want = brute_filter(rho, dc, dims, radius)
        assert np.allclose(got, want, rtol=1e-12, atol=0.0)


def test_oc_update_keeps_volume_bounds_and_move_limit():
    rng = np.random.default_rng(1)
    n = 4000
    rho = rng.uniform(0.05, 0.95, n)
    dc = -rng.lognormal(0.0, 1.5, n)
    for volfrac in (0.4, 0.45, 0.55):  # reachable from a mean of 0.5 within one move
        new = oc_update(rho, dc, volfrac, move=0.2)
        assert abs(new.mean() - volfrac) < 1e-4
        assert np.all(new >= 1e-3) and np.all(new <= 1.0)
        assert np.all(np.abs(new - rho) <= 0.2 + 1e-12)
    # an unreachable target ends at the move limit: every cell as low as it may go
    new = oc_update(rho, dc, 0.1, move=0.2)
    assert np.allclose(new, np.maximum(rho - 0.2, 1e-3), rtol=0, atol=1e-6)


def test_oc_update_moves_material_towards_sensitive_cells():
    """With equal densities, a more negative compliance sensitivity never gets
    less material (the update is rho (-dc / lambda)^eta, clipped)."""
    n = 1000
    rho = np.full(n, 0.4)
    dc = -np.linspace(0.1, 3.0, n)
    new = oc_update(rho, dc, 0.4, move=0.2)
    assert np.all(np.diff(new) >= -1e-15)
    assert new[-1] > new[0]
