"""Z-slab domain decomposition of one field over ranks (one GPU each).

The rows of the (r, Z) grid are split into slabs. A rank's context holds its slab plus two halo
rows on each side that has a neighbour, with the global geometry, frequency grid and inputs
sliced to those rows (lyd_dd_set_halo). Per step:

    colsum <- lyd_dd_step_partials        advection of the owned rows (the stencil reads the halo
                                          rows), emission + frequency step of the owned cells,
                                          and the owned cells' reduction columns
    all-reduce(colsum)                    FindActiveBins energies and the diagnostics' sums
    lyd_dd_finish                         the next window and the step's record, the same on
                                          every rank
    pack / exchange / unpack halos        two rows of J, H_r, H_Z to and from each neighbour

The communication is the caller's: TorchComm uses torch.distributed (NCCL between GPUs, gloo
on the CPU), LocalComm runs every rank's context in one process (one GPU) and does the same
steps with device copies. The kernels never read another GPU's memory.
"""
import copy

import numpy as np

from ._lib import F


def slab_partition(nz, n_ranks):
    """Rows [j0, j1) of each rank: contiguous slabs whose sizes differ by at most one row. Each
    owns at least two rows, so that a neighbour's two halo rows come from one rank."""
    if n_ranks < 1 or nz < 2 * n_ranks:
        raise ValueError(f"{nz} rows cannot be split into {n_ranks} slabs of at least two rows")
    base, extra = divmod(nz, n_ranks)
    out, j = [], 0
    for p in range(n_ranks):
        n = base + (1 if p < extra else 0)
        out.append((j, j + n))
        j += n
    return out


def slab_layout(nz, n_ranks, rank):
    """(j0, j1, h_bot, h_top): the owned rows and the halo rows below and above."""
    j0, j1 = slab_partition(nz, n_ranks)[rank]
    return j0, j1, (2 if rank > 0 else 0), (2 if rank < n_ranks - 1 else 0)


def local_cloud(cloud, j0, j1, h_bot, h_top):
    """The inputs of rows [j0 - h_bot, j1 + h_top) of a workloads.StaticCloud, the geometry
    included (per-row arrays and faces sliced; the boundary intervals apply only at the
    physical boundaries, which keep their global values)."""
    a, b = j0 - h_bot, j1 + h_top
    c = copy.copy(cloud)
    g = copy.copy(cloud.geom)
    g.Z = cloud.geom.Z[a:b + 1]
    g.ZCoM = cloud.geom.ZCoM[a:b]
    for name in ("dV", "inv_dV", "A_r"):
        setattr(g, name, getattr(cloud.geom, name)[a:b])
    g.A_Z = cloud.geom.A_Z[a:b + 1]
    for name in ("dZ_L", "dZ_R", "inv_dZ_j_jm1", "inv_dZ_jp1_j", "inv_dZ_jp2_jp1"):
        setattr(g, name, getattr(cloud.geom, name)[a:b])
    c.geom = g
    for name in ("T", "alpha", "alpha_c", "alpha_cF", "pd", "js", "u_r", "u_Z", "dur_dr", "dur_dZ", "duZ_dr",
                 "duZ_dZ", "ur_over_r", "u_r_star"):
        v = getattr(cloud, name)
        if v is not None and np.ndim(v) == 2:
            setattr(c, name, v[a:b])
    c.u_Z_star = cloud.u_Z_star[a:b + 1]
    if cloud.n_H is not None:
        c.n_H = cloud.n_H[a:b]
    if cloud.species:
        c.species = {k: v[a:b] for k, v in cloud.species.items()}
    return c


class SlabRank:
    """One rank's slab: its context and the device buffers of its communication."""

    def __init__(self, cloud, n_ranks, rank, precision=0, device=0):
        import torch
        from .m1 import context_for_cloud
        self.rank, self.n_ranks = rank, n_ranks
        self.j0, self.j1, self.hb, self.ht = slab_layout(cloud.nz, n_ranks, rank)
        self.cloud = local_cloud(cloud, self.j0, self.j1, self.hb, self.ht)
        self.ctx = context_for_cloud(self.cloud, precision=precision, device=device)
        self.ctx.dd_set_halo(self.hb, self.ht)
        dev = torch.device("cuda", device)
        self.colsum = torch.zeros(self.ctx.dd_columns(), dtype=torch.float64, device=dev)
        sdt = torch.float32 if precision == 2 else torch.float64
        n = 6 * cloud.nr * cloud.n_nu
        mk = lambda: torch.zeros(n, dtype=sdt, device=dev)
        self.send = {0: mk(), 1: mk()}
        self.recv = {0: mk(), 1: mk()}

    def sides(self):
        return [s for s, h in ((0, self.hb), (1, self.ht)) if h]

    def neighbour(self, side):
        return self.rank - 1 if side == 0 else self.rank + 1

    def upload_state(self, J, H_r, H_Z):
        """Global (n_z, n_r, n_nu) arrays: this rank's rows and halo rows of them."""
        a, b = self.j0 - self.hb, self.j1 + self.ht
        for name, v in (("J", J), ("H_r", H_r), ("H_Z", H_Z)):
            self.ctx.upload(name, v[a:b])
            self.ctx.upload(name + "_old", v[a:b])

    def owned(self, name):
        """The owned rows of a downloaded field."""
        v = self.ctx.download(name)
        return v[self.hb:v.shape[0] - self.ht]


class LocalComm:
    """Every rank in this process (one GPU): the all-reduce sums the ranks' column sums, the
    exchange copies each send buffer into the neighbour's receive buffer."""

    def allreduce(self, ranks):
        tot = ranks[0].colsum.clone()
        for r in ranks[1:]:
            tot += r.colsum
        for r in ranks:
            r.colsum.copy_(tot)

    def exchange(self, ranks):
        by = {r.rank: r for r in ranks}
        for r in ranks:
            for s in r.sides():
                r.recv[s].copy_(by[r.neighbour(s)].send[1 - s])


class TorchComm:
    """One rank per process: torch.distributed all-reduce and point-to-point exchange."""

    def allreduce(self, ranks):
        import torch.distributed as dist
        for r in ranks:
            dist.all_reduce(r.colsum)

    def exchange(self, ranks):
        import torch.distributed as dist
        ops = []
        for r in ranks:
            for s in r.sides():
                ops.append(dist.P2POp(dist.isend, r.send[s], r.neighbour(s)))
                ops.append(dist.P2POp(dist.irecv, r.recv[s], r.neighbour(s)))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()


class SlabDriver:
    """Steps the slabs of one field together (the ranks this process holds)."""

    def __init__(self, ranks, comm):
        self.ranks, self.comm = ranks, comm

    def _sync(self):
        import torch
        for r in self.ranks:
            r.ctx.synchronize()
        torch.cuda.synchronize()

    def find_active(self):
        for r in self.ranks:
            r.ctx.dd_find_active_partials(r.colsum)
        self._sync()
        self.comm.allreduce(self.ranks)
        self._sync()
        return [r.ctx.dd_finish(r.colsum, step=False) for r in self.ranks][0]

    def step(self, c_tilde, dt, z_center, bc_r_right, bc_z_bot, bc_z_top):
        for r in self.ranks:
            r.ctx.dd_step_partials(r.colsum, c_tilde, dt, z_center, bc_r_right, bc_z_bot, bc_z_top)
        self._sync()
        self.comm.allreduce(self.ranks)
        self._sync()
        recs = [r.ctx.dd_finish(r.colsum, step=True) for r in self.ranks]
        for r in self.ranks:
            for s in r.sides():
                r.ctx.dd_halo(s, True, r.send[s])
        self._sync()
        self.comm.exchange(self.ranks)
        self._sync()
        for r in self.ranks:
            for s in r.sides():
                r.ctx.dd_halo(s, False, r.recv[s])
        return recs[0]

    def run(self, n_steps, *params):
        self.find_active()
        return np.array([self.step(*params) for _ in range(n_steps)])
