"""NumPy restatement of the learned preconditioner (network, its gradients and
the preconditioner built on it) for small grids.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The preconditioner has no
counterpart in the reference (its solvers are AmgX / AztecOO / Belos); this
file restates the library's own definition so that the CUDA kernels can be
checked:

* network f: four 3x3x3 convolutions on the nodal grid (zero padding),
  5 -> 32 -> 32 -> 32 -> 3 channels, ReLU after the first three; parameters
  as one vector, per layer the weights [out][in][kz][ky][kx] then the biases.
* precision as on the GPU (`bf16=True`): inputs, weights and the outputs of
  layers 1-3 rounded to BF16 (round to nearest even), sums in FP64 here (FP32
  on the tensor cores); the last layer's output is not rounded.
* backward: the gradient of sum(gout . f) with the BF16 roundings treated as
  identity (the weights in the chain are the FP32 parameters, the ReLU masks
  and layer inputs the BF16 activations), as the library's backward kernels do.
* preconditioner: M r = D^-1 r + s D^-1/2 f(D^-1/2 r / s, stiffness,
  Dirichlet), s = sqrt(r.D^-1 r / n_free); stiffness = clip(1 + log10(mean
  diagonal of the node / max over nodes) / 9, 0, 1); Dirichlet = constrained
  fraction of the node's dofs.  Loss of a pair (r, e), K e = r:
  ||e - M r||_K^2 / ||e||_K^2.
"""
import numpy as np

CIN = (5, 32, 32, 32)
COUT = (32, 32, 32, 3)


def num_params():
    return sum(co * ci * 27 + co for ci, co in zip(CIN, COUT))


def unpack(params):
    """Flat parameter vector -> [(W[out, in, kz, ky, kx], b[out]) per layer]."""
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        W = params[o:o + co * ci * 27].reshape(co, ci, 3, 3, 3)
        o += co * ci * 27
        b = params[o:o + co]
        o += co
        out.append((W, b))
    return out


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def conv3(a, W, b):
    """a: (gz, gy, gx, ci); W: (co, ci, 3, 3, 3); out[v] = sum_t W[t] a[v + t - 1] + b (FP64)."""
    gz, gy, gx, _ = a.shape
    p = np.zeros((gz + 2, gy + 2, gx + 2, a.shape[3]))
    p[1:-1, 1:-1, 1:-1] = a
    out = np.zeros((gz, gy, gx, W.shape[0]))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                out += p[dz:dz + gz, dy:dy + gy, dx:dx + gx] @ W[:, :, dz, dy, dx].T.astype(np.float64)
    return out + b


def conv3_input_grad(g, W):
    """Adjoint of conv3 in its input: gin[u] = sum_t W[t]^T g[u - t + 1]."""
    gz, gy, gx, _ = g.shape
    p = np.zeros((gz + 2, gy + 2, gx + 2, g.shape[3]))
    p[1:-1, 1:-1, 1:-1] = g
    out = np.zeros((gz, gy, gx, W.shape[1]))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                out += p[2 - dz:2 - dz + gz, 2 - dy:2 - dy + gy, 2 - dx:2 - dx + gx] @ W[:, :, dz, dy, dx]
    return out


def conv3_weight_grad(g, a):
    """dW[co, ci, t] = sum_v g[v, co] a[v + t - 1, ci]; db = sum_v g."""
    gz, gy, gx, _ = g.shape
    p = np.zeros((gz + 2, gy + 2, gx + 2, a.shape[3]))
    p[1:-1, 1:-1, 1:-1] = a
    dW = np.zeros((g.shape[3], a.shape[3], 3, 3, 3))
    G = g.reshape(-1, g.shape[3])
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                dW[:, :, dz, dy, dx] = G.T @ p[dz:dz + gz, dy:dy + gy, dx:dx + gx].reshape(-1, a.shape[3])
    return dW, G.sum(0)


def forward(params, feat, grid, bf16_round=True):
    """feat: (G, 5) node features, grid = (gx, gy, gz).  Returns (out (G, 3), activations)."""
    gx, gy, gz = grid
    if bf16_round:
        a = bf16(np.asarray(feat, dtype=np.float32)).astype(np.float64)
    else:
        a = np.asarray(feat, dtype=np.float64)
    a = a.reshape(gz, gy, gx, 5)
    acts = [a]
    for l, (W, b) in enumerate(unpack(np.asarray(params, dtype=np.float64))):
        if bf16_round:
            W = bf16(W.astype(np.float32)).astype(np.float64)
            b = b.astype(np.float32).astype(np.float64)
        pre = conv3(a, W, b)
        if l < 3:
            a = np.maximum(pre, 0.0)
            if bf16_round:
                a = bf16(a.astype(np.float32)).astype(np.float64)
            acts.append(a)
        else:
            out = pre
    return out.reshape(-1, 3), acts


def backward(params, feat, grid, gout, bf16_round=True):
    """Gradient of sum(gout . f(feat)) in the parameters (flat vector)."""
    gx, gy, gz = grid
    _, acts = forward(params, feat, grid, bf16_round)
    layers = unpack(np.asarray(params, dtype=np.float64))
    g = np.asarray(gout, dtype=np.float64).reshape(gz, gy, gx, 3)
    grads = [None] * 4
    for l in range(3, -1, -1):
        W, _ = layers[l]
        dW, db = conv3_weight_grad(g, acts[l])
        grads[l] = (dW, db)
        if l > 0:
            g = conv3_input_grad(g, W) * (acts[l] > 0)
    return np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])


def node_features(diag, mask):
    """D^-1, D^-1/2 (interleaved, zero on constrained dofs) and the two node
    features from the interleaved diagonal and the (N,) constrained-dof mask."""
    d = np.asarray(diag, dtype=np.float64).reshape(-1, 3)
    N = d.shape[0]
    c = np.array([[(m >> k) & 1 for k in range(3)] for m in mask], dtype=bool).reshape(N, 3)
    dinv = np.where(c | ~(d > 0), 0.0, 1.0 / np.where(d > 0, d, 1.0))
    m = d.mean(1)
    s = np.clip(1.0 + np.log10(m / m.max()) / 9.0, 0.0, 1.0)
    bc = c.sum(1) / 3.0
    return dinv, np.sqrt(dinv), np.stack([s, bc], 1)


def apply(params, grid, diag, mask, r, bf16_round=True):
    """M r (interleaved 3N vectors)."""
    dinv, dsq, f2 = node_features(diag, mask)
    r = np.asarray(r, dtype=np.float64).reshape(-1, 3)
    nfree = max(1, int((dinv > 0).sum()))
    s = np.sqrt((r * dinv * r).sum() / nfree)
    feat = np.concatenate([r * dsq / s, f2], 1)
    f, _ = forward(params, feat, grid, bf16_round)
    return (dinv * r + s * dsq * f).ravel()


def loss(params, grid, K, diag, mask, r, e, bf16_round=True):
    """||e - M r||_K^2 / ||e||_K^2 with K the constrained (masked) operator."""
    z = apply(params, grid, diag, mask, r, bf16_round)
    d = e - z
    return float(d @ (K @ d) / (e @ (K @ e)))
