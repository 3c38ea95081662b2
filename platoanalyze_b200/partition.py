"""Work partitions for more than one GPU (one process per GPU).

Two ways the cantilever workloads shard:

* independent boxes (the batched workload): each rank solves whole boxes, no
  collective on the data path; `deal_boxes` balances the ranks by the
  estimated work of each box;
* one box cut into slabs along x (`Slabs`): each rank holds the hexes of its
  slab and the nodes on both of its bounding planes; an operator application
  is the local K x of the slab followed by one exchange of the partial sums on
  each interface plane with the neighbouring rank (NCCL send/recv over
  NVLink between GPUs, gloo between CPU processes), and every dot product of
  the CG is a local sum over the nodes the rank owns plus one all-reduce.

The reference distributes a mesh with MPI over Omega_h ghosted partitions
(src/alg/ParallelComm.cpp:49-95, src/PlatoDriver.hpp:77) and sums shared
contributions with its communicator; here the partition is a slab of the
structured box and the exchange moves one plane per neighbour.  The local
operator is a callable (the box kernel of the rank's slab on a GPU), so the
exchange and reduction logic is the same on GPU and CPU ranks.
"""
import numpy as np

# ------------------------------------------------------------- batched boxes --


def box_work(spec):
    """Estimated cost of a Jacobi-PCG solve of an nx x ny x nz cantilever box:
    tets x the longest edge in hexes (the iteration count grows with it)."""
    nx, ny, nz = spec
    return 6 * nx * ny * nz * max(nx, ny, nz)


def deal_boxes(specs, world):
    """Boxes per rank, greedy longest-processing-time first: boxes in order of
    decreasing estimated work, each to the rank with the least work so far
    (ties to the lower rank).  Deterministic; every box on exactly one rank;
    each rank's list in increasing box index.  The largest load is at most
    4/3 of the optimum (Graham's bound) and at most the mean plus one box."""
    order = sorted(range(len(specs)), key=lambda i: (-box_work(specs[i]), i))
    load = [0] * world
    mine = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += box_work(specs[i])
        mine[r].append(i)
    return [sorted(m) for m in mine]


# -------------------------------------------------------------- box slabs --


class Slabs:
    """An nx x ny x nz box (nodes numbered i + px (j + py k)) cut into `world`
    slabs along x: rank r holds hexes [a_r, b_r) and nodes i in [a_r, b_r]
    (interface planes on both ranks that share them); it owns nodes
    i in [a_r, b_r), and the last rank also i = nx."""

    def __init__(self, dims, world, rank):
        nx, ny, nz = dims
        if world > nx:
            raise ValueError("more slabs than hexes along x")
        self.dims, self.world, self.rank = tuple(dims), world, rank
        cuts = [(nx * r) // world for r in range(world + 1)]
        self.a, self.b = cuts[rank], cuts[rank + 1]
        self.px, self.py, self.pz = nx + 1, ny + 1, nz + 1
        self.lpx = self.b - self.a + 1
        self.n_local = self.lpx * self.py * self.pz
        j, k = np.meshgrid(np.arange(self.py), np.arange(self.pz), indexing="ij")
        self._jk = (j + self.py * k).ravel()
        i = np.arange(self.a, self.b + 1)
        # global node of every local node (local numbering i - a + lpx (j + py k))
        ii, jj, kk = np.meshgrid(i, np.arange(self.py), np.arange(self.pz), indexing="ij")
        loc = (ii - self.a) + self.lpx * (jj + self.py * kk)
        self.global_node = np.empty(self.n_local, np.int64)
        self.global_node[loc.ravel()] = (ii + self.px * (jj + self.py * kk)).ravel()
        owned_i = (i < self.b) | (i == nx)
        self.owned = np.zeros(self.n_local, bool)
        self.owned[loc[owned_i].ravel()] = True

    def plane(self, i):
        """Local node ids of the plane at global x index i (a or b)."""
        return (i - self.a) + self.lpx * self._jk

    def local_hexes(self):
        """Global hex ids of the slab in its local hex order (x fastest)."""
        nx, ny, nz = self.dims
        i, j, k = np.meshgrid(np.arange(self.a, self.b), np.arange(ny), np.arange(nz), indexing="ij")
        loc = (i - self.a) + (self.b - self.a) * (j + ny * k)
        g = np.empty(loc.size, np.int64)
        g[loc.ravel()] = (i + nx * (j + ny * k)).ravel()
        return g

    def scatter(self, v_global):
        """The local part of a global interleaved vector (3 per node)."""
        v = np.asarray(v_global).reshape(-1, 3)
        return v[self.global_node].ravel()


class SlabOperator:
    """y = K x for one box distributed as slabs: `local_apply(x_local)` is the
    slab's own operator (interleaved vectors, 3 per local node, any array
    type supporting indexing, e.g. torch tensors on the rank's device); the
    partial sums on the interface planes are exchanged with the neighbours by
    point-to-point messages of 3 py pz values each.  `dist` is
    torch.distributed (initialised by the caller)."""

    def __init__(self, slabs, local_apply, dist, torch):
        self.s, self.local_apply, self.dist, self.torch = slabs, local_apply, dist, torch
        self._left = None if slabs.rank == 0 else self._dof_index(slabs.plane(slabs.a))
        self._right = None if slabs.rank == slabs.world - 1 else self._dof_index(slabs.plane(slabs.b))

    def _dof_index(self, nodes):
        return self.torch.as_tensor((3 * nodes[:, None] + np.arange(3)).ravel(), dtype=self.torch.int64)

    def exchange(self, y):
        """Sum the neighbours' partial sums into the interface planes of y."""
        torch, dist, s = self.torch, self.dist, self.s
        reqs, recv = [], []
        for idx, peer in ((self._left, s.rank - 1), (self._right, s.rank + 1)):
            if idx is None:
                continue
            idx = idx.to(y.device)
            send = y[idx].contiguous()
            buf = torch.empty_like(send)
            reqs.append(dist.isend(send, peer))
            reqs.append(dist.irecv(buf, peer))
            recv.append((idx, buf))
        for r in reqs:
            r.wait()
        for idx, buf in recv:
            y[idx] += buf
        return y

    def __call__(self, x):
        return self.exchange(self.local_apply(x))


def slab_dot(slabs, dist, torch, a, b):
    """Global a . b of two slab-local interleaved vectors: each rank sums its
    owned nodes, one all-reduce."""
    own = torch.as_tensor(np.repeat(slabs.owned, 3), device=a.device)
    t = torch.sum(torch.where(own, a * b, torch.zeros_like(a))).reshape(1)
    dist.all_reduce(t)
    return float(t.item())


def slab_pcg(slabs, op, diag, b, free, dist, torch, rel_tol=1e-10, max_iters=10000):
    """Jacobi-preconditioned CG on the slab-distributed constrained system:
    op (SlabOperator) the unconstrained K, diag its assembled diagonal (after
    the exchange), free a 0/1 mask of the unconstrained dofs (symmetric
    elimination: constrained rows and columns removed), b the right-hand side
    (zero on constrained dofs).  Every rank runs the same iterations; two
    all-reduces per iteration (p . Kp and r . z) plus one for ||r||.
    Returns (x, iterations, relative residual)."""
    x = torch.zeros_like(b)
    dinv = torch.where(free > 0, 1.0 / diag, torch.zeros_like(diag))
    r = b.clone()
    z = dinv * r
    p = z.clone()
    rz = slab_dot(slabs, dist, torch, r, z)
    bb = max(slab_dot(slabs, dist, torch, b, b), 1e-300)
    it = 0
    rr = bb
    while it < max_iters and rr > rel_tol * rel_tol * bb:
        q = op(p * free) * free
        alpha = rz / slab_dot(slabs, dist, torch, p, q)
        x += alpha * p
        r -= alpha * q
        z = dinv * r
        rz_new = slab_dot(slabs, dist, torch, r, z)
        p = z + (rz_new / rz) * p
        rz = rz_new
        rr = slab_dot(slabs, dist, torch, r, r)
        it += 1
    return x, it, (rr / bb) ** 0.5
