"""CPU checks of the learned-preconditioner oracle (oracle/np_net.py): BF16
rounding, the network's backward against central finite differences, and the
training gradient (energy-norm loss through the preconditioner) against
finite differences of the loss."""
import numpy as np

from oracle import np_net, np_ref


def test_bf16_round_to_nearest_even():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 0.0], np.float32)
    got = np_net.bf16(vals)
    want = np.array([1.0, 1.0, 1.0 + 2 * ulp, 1.0, -2.5, 0.0], np.float32)
    assert np.array_equal(got, want)
    assert one == np_net.bf16(one)
    x = np.random.default_rng(0).normal(size=1000).astype(np.float32) * 1e3
    b = np_net.bf16(x)
    assert not (b.view(np.uint32) & 0xFFFF).any()
    half_ulp = np.ldexp(np.float32(1.0), np.frexp(np.abs(x))[1] - 9)
    assert (np.abs(b - x) <= half_ulp).all()


def _params(rng, scale_last=0.3):
    p = np.zeros(np_net.num_params())
    o = 0
    for ci, co in zip(np_net.CIN, np_net.COUT):
        n = co * ci * 27
        p[o:o + n] = rng.normal(0.0, np.sqrt(2.0 / (27 * ci)), n) * (scale_last if co == 3 else 1.0)
        o += n
        p[o:o + co] = rng.normal(0.0, 0.05, co)
        o += co
    return p


def test_parameter_count():
    assert np_net.num_params() == 62307


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    grid = (4, 3, 3)
    G = 36
    p = _params(rng)
    feat = rng.normal(size=(G, 5))
    gout = rng.normal(size=(G, 3))
    g = np_net.backward(p, feat, grid, gout, bf16_round=False)

    def L(q):
        return float((np_net.forward(q, feat, grid, bf16_round=False)[0] * gout).sum())

    idx = np.concatenate([rng.choice(np_net.num_params(), 24, replace=False), [0, np_net.num_params() - 1]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (L(p + e) - L(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def _small_problem(rng):
    nx, ny, nz = 3, 2, 2
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    z = np.repeat(rng.uniform(0.2, 1.0, nx * ny * nz), 6)
    prob = np_ref.Problem(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    K = prob.stiffness_dense(z)
    N = coords.shape[0]
    clamp = np.where(coords[:, 0] < 1e-9)[0]
    mask = np.zeros(N, np.uint8)
    mask[clamp] = 7
    free = np.repeat(mask == 0, 3)
    Km = K * np.outer(free, free)
    return (nx + 1, ny + 1, nz + 1), np.diag(K).copy(), mask, Km, free


def test_training_gradient_matches_finite_differences():
    """dL/dparams by the chain the training kernels use:
    dL/dz = 2 (K z - r) / (e.r), dL/df = s D^-1/2 dL/dz, then the network backward."""
    rng = np.random.default_rng(5)
    grid, diag, mask, Km, free = _small_problem(rng)
    e = rng.normal(size=Km.shape[0]) * free
    r = Km @ e
    p = _params(rng)

    def loss(q):
        return np_net.loss(q, grid, Km, diag, mask, r, e, bf16_round=False)

    dinv, dsq, f2 = np_net.node_features(diag, mask)
    R = r.reshape(-1, 3)
    s = np.sqrt((R * dinv * R).sum() / free.sum())
    z = np_net.apply(p, grid, diag, mask, r, bf16_round=False)
    dz = 2.0 * (Km @ z - r) / (e @ r)
    gout = s * dsq * dz.reshape(-1, 3)
    feat = np.concatenate([R * dsq / s, f2], 1)
    g = np_net.backward(p, feat, grid, gout, bf16_round=False)
    h = 1e-6
    for i in np.concatenate([rng.choice(np_net.num_params(), 20, replace=False), [np_net.num_params() - 2]]):
        ei = np.zeros_like(p)
        ei[i] = h
        fd = (loss(p + ei) - loss(p - ei)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd)), (i, fd, g[i])


def test_zero_last_layer_is_jacobi():
    rng = np.random.default_rng(7)
    grid, diag, mask, Km, free = _small_problem(rng)
    p = _params(rng, scale_last=0.0)
    last_b = np_net.num_params() - 3
    p[last_b:] = 0.0
    r = rng.normal(size=Km.shape[0]) * free
    z = np_net.apply(p, grid, diag, mask, r)
    dinv, _, _ = np_net.node_features(diag, mask)
    assert np.allclose(z, (dinv.ravel() * r), rtol=0, atol=1e-14)
    # the loss of Jacobi is below 1 (one Jacobi step reduces the energy error)
    e = np.linalg.lstsq(Km + np.diag(~free * 1.0), r, rcond=None)[0]
    assert 0.0 < np_net.loss(p, grid, Km, diag, mask, r, e) < 1.0
