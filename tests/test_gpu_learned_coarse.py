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
    lc.attach(prob)
    u1, s1 = prob.solution(z, options=opts)
    assert s1["iterations"] == s0["iterations"]
    assert torch.equal(u0, u1)
    prob.set_coarse_network(None)
    assert float(lc.delta(prob, z).abs().max()) == 0.0
    lc.close()


def test_trained_coarse_network_selected_by_cg_iterations(pa):
    """32^3 SIMP cantilever: residual/error pairs from multigrid solves of
    design iterations 8-29, Adam on the V-cycle's energy-norm loss, the CG
    iterations on the last training design counted every 20 steps.  The loss
    falls; the parameters kept are those with the fewest CG iterations, the
    untrained network (the plain multigrid) unless a checkpoint beats it, and
    the solve of the held-out final design stays correct.  Measured on these
    designs: 96 iterations untrained, 105-110 at every checkpoint, so the
    untrained network is kept and the trained correction gains nothing."""
    import torch
    from platoanalyze_b200.api import LearnedCoarsening
    from platoanalyze_b200.workloads import cantilever, simp_training_pairs
    dims = (32, 32, 32)
    mesh, prob, faces, dofs = cantilever(dims)
    dens, sd, res, en, final, hist = simp_training_pairs(prob, dims, iterations=30, snapshots=(2, 4, 8, 16),
                                                         solver="mg", first=8)
    assert len(sd) >= 60
    lc = LearnedCoarsening(prob, seed=0)
    zf = torch.tensor(final, device="cuda")
    plain = lc.iterations(prob, zf)
    tr = lc.train(prob, dens, res, en, sd, steps=100, batch=4, learning_rate=3e-3, seed=1, validation=dens[-1],
                  check_every=20)
    loss = np.array(tr["loss"])
    assert np.all(np.isfinite(loss)) and loss[-20:].mean() < loss[:20].mean()
    checks = dict(tr["iterations"])
    untrained = checks[0]
    kept = checks[tr["kept_step"]]
    assert kept == min(checks.values()) and kept <= untrained
    held_out = lc.iterations(prob, zf)
    if tr["kept_step"] == 0:
        # delta is exactly zero again: the plain method, whose count moves by
        # an iteration or two with the warm-started spectral estimate (the
        # problem solved other designs in between)
        assert abs(held_out - plain) <= 2, (checks, held_out, plain)
    lc.attach(prob)
    u, st = prob.solution(zf, options=pa.SolveOptions("mg", rel_tol=1e-8))
    prob.set_coarse_network(None)
    u64, _ = prob.solution(zf, options=pa.SolveOptions("fp64", rel_tol=1e-10))
    f = prob.scalar_function().value(u, zf)
    f64 = prob.scalar_function().value(u64, zf)
    assert st["converged"] and abs(f - f64) <= 1e-6 * abs(f64)
    lc.close()
