"""NumPy FP64 restatement of the linear-tet SIMP elastostatics path.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Plain loops over cells;
meant for meshes of at most a few thousand tets.  Each function cites the
reference lines it restates (paths relative to the platoanalyze tree).
"""
import numpy as np

# Six tets of one hex, vertex offsets and local order as in the reference's
# single-hex box (unit_tests/OmegaHUtilitiesTests.cpp:258-287).
HEX_TETS = (
    ((0, 0, 0), (1, 1, 0), (0, 1, 0), (1, 1, 1)),
    ((0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1)),
    ((0, 0, 0), (0, 1, 1), (0, 0, 1), (1, 1, 1)),
    ((0, 0, 0), (1, 0, 1), (1, 1, 1), (0, 0, 1)),
    ((1, 0, 0), (1, 0, 1), (1, 1, 1), (0, 0, 0)),
    ((1, 0, 0), (1, 1, 1), (1, 1, 0), (0, 0, 0)),
)


def box_mesh(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0):
    """Nodes x-fastest, hexes x-fastest, 6 tets per hex (HEX_TETS order)."""
    px, py = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    coords = np.stack([lx * i.ravel() / nx, ly * j.ravel() / ny, lz * k.ravel() / nz], axis=1).astype(np.float64)
    hk, hj, hi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    cells = np.empty((hi.size, 6, 4), dtype=np.int32)
    for t, tet in enumerate(HEX_TETS):
        for n, (a, b, c) in enumerate(tet):
            cells[:, t, n] = (hi + a) + px * ((hj + b) + py * (hk + c))
    return cells.reshape(-1, 4), coords


def boundary_faces(cells, coords, axis, value, tol=1e-12):
    """Tet faces whose three vertices lie on the plane x[axis] == value."""
    faces = []
    on = np.abs(coords[:, axis] - value) <= tol
    for c in cells:
        for drop in range(4):
            f = [c[n] for n in range(4) if n != drop]
            if on[f].all():
                faces.append(f)
    return np.array(faces, dtype=np.int32).reshape(-1, 3)


def stiffness(E, nu):
    """IsotropicLinearElasticMaterial<3> (src/IsotropicLinearElasticMaterial.cpp:86-108)."""
    c = E / ((1 + nu) * (1 - 2 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = c * nu
    for i in range(3):
        C[i, i] = c * (1 - nu)
        C[i + 3, i + 3] = 0.5 * c * (1 - 2 * nu)
    return C


def cell_gradients(X):
    """ComputeGradientWorkset<3> (src/ImplicitFunctors.hpp:165-217) x weight 1/6."""
    J = np.array([[X[n][d] - X[3][d] for n in range(3)] for d in range(3)])
    inv = np.linalg.inv(J)
    g = np.zeros((4, 3))
    g[:3] = inv
    g[3] = -inv.sum(0)
    return g, abs(np.linalg.det(J)) / 6.0


def bmatrix(g):
    """Strain<3> (src/Strain.hpp:56-94) as a 6x12 matrix, Voigt xx,yy,zz,yz,xz,xy."""
    B = np.zeros((6, 12))
    for n in range(4):
        for d in range(3):
            B[d, 3 * n + d] = g[n, d]
        B[3, 3 * n + 1], B[3, 3 * n + 2] = g[n, 2], g[n, 1]
        B[4, 3 * n + 0], B[4, 3 * n + 2] = g[n, 2], g[n, 0]
        B[5, 3 * n + 0], B[5, 3 * n + 1] = g[n, 1], g[n, 0]
    return B


def simp(rho, p, pmin):
    """MSIMP (src/Simp.hpp:130-134)."""
    return pmin + (1 - pmin) * rho ** p


def simp_deriv(rho, p, pmin):
    return (1 - pmin) * p * rho ** (p - 1) if rho != 0 else ((1 - pmin) if p == 1 else 0.0)


def cell_rho(z, cell, c, layout):
    return z[c] if layout == 1 else z[cell].mean()


class Problem:
    """Small-case restatement of Elliptic::VectorFunction / PhysicsScalarFunction."""

    def __init__(self, cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=0):
        self.cells = np.asarray(cells, dtype=np.int32)
        self.coords = np.asarray(coords, dtype=np.float64)
        self.N = self.coords.shape[0]
        self.C = self.cells.shape[0]
        self.Cm = stiffness(E, nu)
        self.p, self.pmin, self.layout = p, pmin, layout
        self.geo = [cell_gradients(self.coords[c]) for c in self.cells]

    def cell_k(self, c):
        g, v = self.geo[c]
        B = bmatrix(g)
        return v * B.T @ self.Cm @ B

    def dofs(self, c):
        return np.array([3 * a + d for a in self.cells[c] for d in range(3)])

    def stiffness_dense(self, z):
        K = np.zeros((3 * self.N, 3 * self.N))
        for c in range(self.C):
            w = simp(cell_rho(z, self.cells[c], c, self.layout), self.p, self.pmin)
            idx = self.dofs(c)
            K[np.ix_(idx, idx)] += w * self.cell_k(c)
        return K

    def traction(self, faces, flux):
        """SurfaceLoadIntegral (src/SurfaceLoadIntegral.hpp:96-160), scale +1."""
        F = np.zeros(3 * self.N)
        for f in faces:
            a = self.coords[f[0]] - self.coords[f[2]]
            b = self.coords[f[1]] - self.coords[f[2]]
            w = np.linalg.norm(np.cross(a, b)) / 6.0
            for n in f:
                F[3 * n:3 * n + 3] += w * np.asarray(flux)
        return F

    def value(self, u, z, faces=None, flux=None):
        """VectorFunction::value: K(z) u - F."""
        r = self.stiffness_dense(z) @ u
        if faces is not None and len(faces):
            r -= self.traction(faces, flux)
        return r

    def gradient_z_dense(self, u, z):
        """dR/dz as a dense (nz x 3N) matrix (transposed Jacobian layout)."""
        nz = self.C if self.layout == 1 else self.N
        G = np.zeros((nz, 3 * self.N))
        for c in range(self.C):
            cell = self.cells[c]
            rho = cell_rho(z, cell, c, self.layout)
            dw = simp_deriv(rho, self.p, self.pmin)
            idx = self.dofs(c)
            re = self.cell_k(c) @ u[idx]
            if self.layout == 1:
                G[c, idx] += dw * re
            else:
                for k in cell:
                    G[k, idx] += 0.25 * dw * re
        return G

    def energy(self, u, z):
        """InternalElasticEnergy value, gradient_u, gradient_z."""
        f = 0.0
        gu = np.zeros(3 * self.N)
        gz = np.zeros(self.C if self.layout == 1 else self.N)
        for c in range(self.C):
            cell = self.cells[c]
            rho = cell_rho(z, cell, c, self.layout)
            w, dw = simp(rho, self.p, self.pmin), simp_deriv(rho, self.p, self.pmin)
            idx = self.dofs(c)
            ke = self.cell_k(c)
            e0 = 0.5 * u[idx] @ ke @ u[idx]
            f += w * e0
            gu[idx] += w * ke @ u[idx]
            if self.layout == 1:
                gz[c] += dw * e0
            else:
                gz[cell] += 0.25 * dw * e0
        return f, gu, gz


def crs_graph(cells, N):
    """Node-star graph with diagonal, columns sorted ascending."""
    adj = [set() for _ in range(N)]
    for c in cells:
        for a in c:
            adj[a].update(int(b) for b in c)
    rowmap = np.zeros(N + 1, dtype=np.int32)
    cols = []
    for i in range(N):
        s = sorted(adj[i])
        cols += s
        rowmap[i + 1] = rowmap[i] + len(s)
    return rowmap, np.array(cols, dtype=np.int32)


def block_entries(K, rowmap, cols, bi=3, bj=3):
    """Pack a dense matrix into block-CRS entry order [block][i][j]."""
    out = []
    for r in range(len(rowmap) - 1):
        for k in range(rowmap[r], rowmap[r + 1]):
            c = cols[k]
            out.append(K[bi * r:bi * r + bi, bj * c:bj * c + bj].ravel())
    return np.concatenate(out)
