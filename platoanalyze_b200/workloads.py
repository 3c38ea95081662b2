"""Synthetic workloads: the SIMP cantilever boxes the benchmark and tests use.

A box of nx x ny x nz unit hexes, each split into 6 linear tets (the mesh of
pa_mesh_create_box), clamped on x = 0 (all three dofs of every node there),
loaded by a uniform traction of unit total magnitude on the x = nx face.
Densities are per hex (all 6 tets of a hex share it), either i.i.d. uniform
or a Gaussian-smoothed random field.  No dataset is involved; every field is
generated from a seed.
"""
import numpy as np

from .api import Mesh, Problem

CONFIGS = {
    # 20x10x10 hexes, i.i.d. U[0.3, 1] densities, FP64 Jacobi-PCG to 1e-10
    "cantilever_20x10x10_fp64": dict(dims=(20, 10, 10), density="uniform", lo=0.3, hi=1.0, rel_tol=1e-10,
                                     method="fp64"),
    # 160x80x80 hexes (6,144,000 tets), smoothed field clipped to [0.01, 1], mixed precision to 1e-8
    "cantilever_160x80x80_mixed": dict(dims=(160, 80, 80), density="smoothed", sigma=3.0, lo=0.01, hi=1.0,
                                       rel_tol=1e-8, method="mixed"),
}


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


def cantilever(dims, youngs_modulus=1.0, poissons_ratio=0.3, simp_exponent=3.0, simp_min=1e-9, stream=None):
    """Mesh + Problem (per-cell controls) with the clamp and the end traction."""
    nx, ny, nz = dims
    mesh = Mesh.box(nx, ny, nz, float(nx), float(ny), float(nz))
    prob = Problem(mesh, youngs_modulus, poissons_ratio, simp_exponent, simp_min, control_layout="cell",
                   stream=stream)
    faces = mesh.boundary_faces(0, float(nx))
    prob.add_traction(faces, np.array([0.0, 0.0, -1.0 / (ny * nz)]))
    # x = 0 nodes of the x-fastest numbering: i = 0
    px, py = nx + 1, ny + 1
    jj, kk = np.meshgrid(np.arange(py), np.arange(nz + 1), indexing="ij")
    nodes = (px * (jj + py * kk)).ravel()
    dofs = np.sort(np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2])).astype(np.int32)
    prob.set_dirichlet(dofs)
    return mesh, prob, faces, dofs
