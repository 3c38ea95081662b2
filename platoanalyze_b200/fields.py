"""Synthetic density fields and box meshes of the SIMP cantilever workloads.

NumPy/SciPy only: this module never loads libpa_b200.so, so a CPU-only
process (the timed CPU baseline of the same workload) can import it by path
without importing the package.

A box of nx x ny x nz unit hexes is split into 6 linear tets per hex (the
split of pa_mesh_create_box), nodes and hexes numbered x fastest.  Densities
are per hex (all 6 tets of a hex share it), either i.i.d. uniform or a
Gaussian-smoothed random field.  No dataset is involved; every field is
generated from a seed.
"""
import numpy as np

# Six tets of a unit hex (vertex offsets), the split of pa_mesh_create_box:
# the six paths from corner (0,0,0) to (1,1,1) along the three axes.
HEX_TETS = (
    ((0, 0, 0), (1, 1, 0), (0, 1, 0), (1, 1, 1)),
    ((0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1)),
    ((0, 0, 0), (0, 1, 1), (0, 0, 1), (1, 1, 1)),
    ((0, 0, 0), (1, 0, 1), (1, 1, 1), (0, 0, 1)),
    ((1, 0, 0), (1, 0, 1), (1, 1, 1), (0, 0, 0)),
    ((1, 0, 0), (1, 1, 1), (1, 1, 0), (0, 0, 0)),
)


def hex_density(dims, seed, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0):
    """Per-hex density on the (nz, ny, nx) grid, flattened x fastest.

    smoothed: white noise U[0,1] (numpy PCG64, `seed`), separable Gaussian
    filter with sigma cells truncated at 3 sigma (reflecting borders), affine
    rescale to [0, 1], clip to [lo, hi].  uniform: i.i.d. U[lo, hi]."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.uniform(lo, hi, nx * ny * nz)
    from scipy.ndimage import gaussian_filter
    noise = rng.uniform(0.0, 1.0, (nz, ny, nx))
    f = gaussian_filter(noise, sigma=sigma, truncate=3.0, mode="reflect")
    f = (f - f.min()) / max(f.max() - f.min(), 1e-300)
    return np.clip(f, lo, hi).ravel()


def cell_density(dims, seed, **kw):
    """Per-tet density: each hex value repeated for its 6 tets."""
    return np.repeat(hex_density(dims, seed, **kw), 6)


def box_arrays(nx, ny, nz):
    """Connectivity (C x 4, int32), coordinates (N x 3, unit hexes), the
    triangles of the x = nx face (tets 4 and 5 of the last hex column) and the
    nodes of the x = 0 face, in the numbering of pa_mesh_create_box."""
    px, py = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    coords = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    hk, hj, hi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    cells = np.empty((hi.size, 6, 4), dtype=np.int32)
    for t, tet in enumerate(HEX_TETS):
        for n, (a, b, c) in enumerate(tet):
            cells[:, t, n] = (hi + a) + px * ((hj + b) + py * (hk + c))
    last = hi == nx - 1
    node = lambda a, b, c: (hi[last] + a) + px * ((hj[last] + b) + py * (hk[last] + c))
    faces = np.concatenate([np.stack([node(1, 0, 0), node(1, 0, 1), node(1, 1, 1)], 1),
                            np.stack([node(1, 0, 0), node(1, 1, 1), node(1, 1, 0)], 1)]).astype(np.int32)
    jj, kk = np.meshgrid(np.arange(py), np.arange(nz + 1), indexing="ij")
    clamp = (px * (jj + py * kk)).ravel()
    return cells.reshape(-1, 4), coords, faces, clamp


def clamp_dofs(clamp):
    """All three dofs of the clamped nodes, sorted (int32)."""
    clamp = np.asarray(clamp, np.int64)
    return np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
