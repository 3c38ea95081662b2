"""Learned level-1 weights of the box multigrid (pa_boxmg_coarse_*,
pa_problem_set_coarse_network): the loss gradient against central
differences on a two-level hierarchy (where it is exact), a new network
leaving the method unchanged, and a network trained on SIMP residual/error
pairs against the untrained one on a design it did not see."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs(prob, z, dofs, n, count, seed):
    import torch
    rng = np.random.default_rng(seed)
    R, E = [], []
    for _ in range(count):
        e = torch.tensor(rng.standard_normal(3 * n), device="cuda")
        e[torch.as_tensor(dofs, device="cuda").long()] = 0.0
        r = prob.apply(z, e, constrained=True)
        R.append(r)
        E.append(float(torch.dot(e, r)))
    return torch.stack(R), E


def test_coarse_sensitivity_matches_central_differences(pa):
    """8x4x4 hexes: level 1 (4x2x2) is the coarsest and solved exactly, so
    dloss/ddelta is the exact derivative of the V-cycle's energy-norm loss."""
    import torch
    from platoanalyze_b200.workloads import cantilever, cell_density
    dims = (8, 4, 4)
    mesh, prob, faces, dofs = cantilever(dims)
    z = torch.tensor(cell_density(dims, 3, kind="smoothed", sigma=1.0, lo=0.001, hi=1.0), device="cuda")
    g1 = prob.coarse_grid()
    assert g1 == (4, 2, 2)
    H1 = g1[0] * g1[1] * g1[2]
    R, E = _pairs(prob, z, dofs, mesh.num_nodes, 3, 0)
    rng = np.random.default_rng(1)
    delta = torch.tensor(0.3 * rng.standard_normal(H1), dtype=torch.float32, device="cuda")
    for _ in range(6):  # settle the warm-started spectral estimate of the fine smoother
        prob.coarse_sensitivity(z, delta, R, E)
    loss, g = prob.coarse_sensitivity(z, delta, R, E)
    g = g.clone()
    assert 0.0 < loss < 1.0
    for i in (0, 5, H1 - 1):
        h = 0.05
        dp, dm = delta.clone(), delta.clone()
        dp[i] += h
        dm[i] -= h
        fd = (prob.coarse_sensitivity(z, dp, R, E)[0] - prob.coarse_sensitivity(z, dm, R, E)[0]) / (2 * h)
        assert abs(fd - float(g[i])) <= 0.03 * abs(fd) + 1e-4 * float(g.abs().max()), (i, fd, float(g[i]))
    d = torch.tensor(rng.standard_normal(H1), dtype=torch.float32, device="cuda")
    fd = (prob.coarse_sensitivity(z, delta + 0.02 * d, R, E)[0] -
          prob.coarse_sensitivity(z, delta - 0.02 * d, R, E)[0]) / 0.04
    assert abs(fd - float(torch.dot(g, d))) <= 0.03 * abs(fd)


def test_new_coarse_network_is_the_plain_multigrid(pa):
    """A new network (last layer zero) gives delta = 0: a fresh problem with it
    attached takes the same iterations to the same solution bits as a fresh
    problem without it."""
    import torch
    from platoanalyze_b200.api import LearnedCoarsening
    from platoanalyze_b200.workloads import cantilever, cell_density
    dims = (16, 8, 8)
    _, prob0, _, _ = cantilever(dims)
    mesh, prob, faces, dofs = cantilever(dims)
    z = torch.tensor(cell_density(dims, 5, kind="smoothed", sigma=1.5, lo=0.01, hi=1.0), device="cuda")
    opts = pa.SolveOptions("mg", rel_tol=1e-10)
    u0, s0 = prob0.solution(z, options=opts)
    lc = LearnedCoarsening(prob, seed=3)
    assert lc.grid == (8, 4, 4)
    assert float(lc.delta(prob, z).abs().max()) == 0.0
    lc.attach(prob)
    u1, s1 = prob.solution(z, options=opts)
    assert s1["iterations"] == s0["iterations"]
    assert torch.equal(u0, u1)
    prob.set_coarse_network(None)
    lc.close()
