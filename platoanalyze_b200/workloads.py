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
from .fields import HEX_TETS, box_arrays, cell_density, hex_density  # noqa: F401  (re-exported)

CONFIGS = {
    # 20x10x10 hexes, i.i.d. U[0.3, 1] densities, FP64 Jacobi-PCG to 1e-10
    "cantilever_20x10x10_fp64": dict(dims=(20, 10, 10), density="uniform", lo=0.3, hi=1.0, rel_tol=1e-10,
                                     method="fp64"),
    # 160x80x80 hexes (6,144,000 tets), smoothed field clipped to [0.01, 1], multigrid CG to 1e-8
    "cantilever_160x80x80_mg": dict(dims=(160, 80, 80), density="smoothed", sigma=3.0, lo=0.01, hi=1.0,
                                    rel_tol=1e-8, method="mg"),
}


def cantilever(dims, youngs_modulus=1.0, poissons_ratio=0.3, simp_exponent=3.0, simp_min=1e-9, stream=None,
               uniform_geometry=True):
    """Mesh + Problem (per-cell controls) with the clamp and the end traction.
    uniform_geometry=False makes the FP32 kernels recompute the geometry per
    tet instead of reading the box's hex geometry table."""
    nx, ny, nz = dims
    mesh = Mesh.box(nx, ny, nz, float(nx), float(ny), float(nz))
    if not uniform_geometry:
        mesh.set_uniform_geometry(False)
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


# ------------------------------------------------------------------------------
# SIMP design iterations and (residual, error) pairs for the learned
# preconditioner.  The optimality-criteria update belongs to the optimizer that
# drives Plato Analyze (Plato Engine, not part of the reference); it is written
# here from the published method (Bendsoe & Sigmund: OC with bisection on the
# volume multiplier, move limit, damping 1/2, sensitivity filter of radius
# 1.5 hexes) only to produce the densities the pairs come from.

def sensitivity_filter(rho, dc, dims, radius=1.5):
    """Mesh-independency filter on the hex grid: dc_i = sum_j H_ij rho_j dc_j /
    (max(rho_i, 1e-3) sum_j H_ij), H_ij = max(0, radius - dist(i, j))."""
    from scipy.ndimage import correlate
    nx, ny, nz = dims
    r = int(np.floor(radius))
    ax = np.arange(-r, r + 1)
    dz, dy, dx = np.meshgrid(ax, ax, ax, indexing="ij")
    H = np.maximum(0.0, radius - np.sqrt(dx ** 2 + dy ** 2 + dz ** 2))
    g = lambda a: a.reshape(nz, ny, nx)
    num = correlate(g(rho * dc), H, mode="constant")
    den = correlate(np.ones((nz, ny, nx)), H, mode="constant")
    return (num / (np.maximum(g(rho), 1e-3) * den)).ravel()


def oc_update(rho, dc, volfrac, move=0.2, eta=0.5, rho_min=1e-3):
    """Optimality-criteria update with bisection on the volume multiplier."""
    lo, hi = 1e-12, 1e12
    dc = np.minimum(dc, -1e-300)
    new = rho
    while (hi - lo) / (hi + lo) > 1e-7:
        lam = np.sqrt(lo * hi)
        new = rho * (-dc / lam) ** eta
        new = np.clip(new, np.maximum(rho - move, rho_min), np.minimum(rho + move, 1.0))
        if new.mean() > volfrac:
            lo = lam
        else:
            hi = lam
    return new


def simp_training_pairs(prob, dims, iterations=30, snapshots=(8, 32, 128, 512), volfrac=0.4, move=0.2,
                        check_every=64, device="cuda", log=None, solver="mixed", first=0):
    """Run `iterations` SIMP/OC design iterations on the cantilever; at each,
    the plain solve (solver "mixed": Jacobi-PCG; "mg": the box multigrid CG)
    to 1e-10 gives u*, and the iterates x_k of plain solves stopped after k in
    `snapshots` iterations give the pairs e = u* - x_k, r = K e (constrained
    operator), E = e . r; pairs are taken from design iteration `first` on.

    Returns (densities [n_it x C], sample_density, residuals [n_s x 3N],
    energies, final_density, history) with the big arrays as torch tensors on
    `device`; final_density is the OC update after the last iteration (a
    design the pairs did not see)."""
    import torch
    from .api import SolveOptions
    nx, ny, nz = dims
    H = nx * ny * nz
    rho = np.full(H, volfrac)
    dens, sd, res, en, hist = [], [], [], [], []
    plain = SolveOptions(solver, rel_tol=1e-10, check_every=check_every)
    for it in range(iterations):
        zc = torch.tensor(np.repeat(rho, 6), device=device)
        u, st = prob.solution(zc, options=plain)
        c = prob.scalar_function().value(u, zc)
        g = prob.criterion_gradient(zc, u)  # compliance sensitivity at equilibrium (<= 0), per cell
        dc = g.view(-1, 6).sum(1).cpu().numpy()
        dens.append(zc)
        for k in (snapshots if it >= first else ()):
            xk, _ = prob.solution(zc, options=SolveOptions(solver, rel_tol=1e-14, max_iters=k,
                                                           check_every=check_every), allow_not_converged=True)
            e = u - xk
            r = prob.apply(zc, e, constrained=True)
            E = float(torch.dot(e, r).item())
            if E > 0.0:
                res.append(r)
                en.append(E)
                sd.append(it)
        hist.append({"iteration": it, "compliance": c, "cg_iterations": st["iterations"],
                     "volume": float(rho.mean())})
        if log:
            log(hist[-1])
        dc = sensitivity_filter(rho, dc, dims)
        rho = oc_update(rho, dc, volfrac, move)
    return (torch.stack(dens), np.array(sd, np.int32), torch.stack(res), np.array(en), np.repeat(rho, 6), hist)


# ------------------------------------------------------------------------------
# Batched boxes: many independent cantilevers solved side by side on one
# parted mesh (one CG per box).

def _box(nx, ny, nz):
    return box_arrays(nx, ny, nz)


def batch_specs(count=64, seed=1234, lo=16, hi=48):
    """Box sizes U{lo..hi}^3 and unit traction directions (uniform on the
    sphere) from one seed; box i's density uses seed + i."""
    rng = np.random.default_rng(seed)
    dims = rng.integers(lo, hi + 1, size=(count, 3))
    d = rng.normal(size=(count, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return [tuple(int(v) for v in row) for row in dims], d


def batched_boxes(specs, directions, seed=1234, stream=None, sigma=3.0, box_ids=None):
    """One parted mesh + Problem holding every box (each clamped at its x = 0
    face, unit total traction along its direction on its x = max face) and
    the per-cell densities (smoothed field, seed + i, or seed + box_ids[i]
    when the boxes are a subset of a larger batch).  Boxes are laid out
    along x with a gap, parts = boxes."""
    cells_l, coords_l, z_l, faces_l, clamp_l, offs = [], [], [], [], [], [0]
    x0, nn = 0.0, 0
    for i, (nx, ny, nz) in enumerate(specs):
        c, X, f, cl = _box(nx, ny, nz)
        X[:, 0] += x0
        cells_l.append(c + nn)
        coords_l.append(X)
        faces_l.append(f + nn)
        clamp_l.append(cl + nn)
        bid = i if box_ids is None else int(box_ids[i])
        z_l.append(cell_density((nx, ny, nz), seed + bid, kind="smoothed", sigma=sigma, lo=0.01, hi=1.0))
        nn += X.shape[0]
        offs.append(nn)
        x0 += nx + 4.0
    mesh = Mesh.from_arrays(np.concatenate(cells_l), np.concatenate(coords_l))
    mesh.set_parts(np.array(offs, np.int64))
    prob = Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell", stream=stream)
    for (nx, ny, nz), f, d in zip(specs, faces_l, directions):
        prob.add_traction(f, np.asarray(d, np.float64) / (ny * nz))
    clamp = np.concatenate(clamp_l)
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    prob.set_dirichlet(dofs)
    return mesh, prob, np.concatenate(z_l), np.array(offs, np.int64)
