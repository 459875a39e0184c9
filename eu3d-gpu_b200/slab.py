"""One grid decomposed along x over ranks, one x block per rank.

The reference's MPI layout with m_block_x = ranks (Mesh::Initial,
src/Mesh.cpp:96-119: block r holds global nodes r (n - 1) .. r (n - 1) + n - 1
with n = (total_ni - 1) / ranks + 1, so neighbouring blocks share one node),
its halo exchange before each step (Flowfield::Mpi_Boundary,
src/Flowfield.cpp:809-911: the bc node planes next to a shared node go to the
neighbour's ghost planes) and the CFL minimum over blocks
(Flowfield::CFLcondition's MPI_Allreduce(MPI_MIN), src/Flowfield.cpp:275-304).
Messages move with torch.distributed point-to-point operations: NCCL between
GPUs, gloo between CPU processes.

    block_range(total_ni, ranks, rank)  -> (first global node, nodes)
    HaloExchange(dist, rank, ranks, ...) -> moves one step's messages
    SlabSolver(dist, grid, extent, ...)  -> an eu3d.Solver on this rank's block
"""
from __future__ import annotations

import numpy as np

import eu3d


def block_range(total_ni, blocks, block):
    """First global node and node count of x block `block` of `blocks`."""
    if blocks < 1 or not 0 <= block < blocks or (total_ni - 1) % blocks:
        raise ValueError(f"{total_ni} nodes do not split into {blocks} x blocks (total_ni - 1 must divide)")
    n = (total_ni - 1) // blocks + 1
    return block * (n - 1), n


def block_slice(a, total_ni, blocks, block, bc=2, axis=-3):
    """The haloed planes of block `block` out of a global haloed array: global
    node g sits at haloed index g + bc, so the block's haloed planes are
    first .. first + n + 2 bc - 1 (its internal-face ghost planes hold the
    neighbours' nodes, as after an exchange)."""
    first, n = block_range(total_ni, blocks, block)
    idx = [slice(None)] * a.ndim
    idx[axis] = slice(first, first + n + 2 * bc)
    return a[tuple(idx)]


class HaloExchange:
    """The halo messages of one block and its x neighbours (rank r holds
    block r). exchange(pack, unpack): pack(face, buf) fills the outgoing
    message of face 0 (x low, to rank - 1) or 1 (x high, to rank + 1),
    unpack(face, buf) consumes the incoming one; the four transfers of a step
    go out as one batch of point-to-point operations."""

    def __init__(self, dist, rank, ranks, numel, dtype, device):
        import torch
        self.dist, self.rank, self.ranks = dist, rank, ranks
        faces = [f for f, peer in ((0, rank - 1), (1, rank + 1)) if 0 <= peer < ranks]
        self.peers = {0: rank - 1, 1: rank + 1}
        self.faces = faces
        self.send = {f: torch.empty(numel, dtype=dtype, device=device) for f in faces}
        self.recv = {f: torch.empty(numel, dtype=dtype, device=device) for f in faces}

    def exchange(self, pack, unpack):
        if not self.faces:
            return
        dist = self.dist
        ops = []
        for f in self.faces:
            pack(f, self.send[f])
            ops.append(dist.P2POp(dist.isend, self.send[f], self.peers[f]))
            ops.append(dist.P2POp(dist.irecv, self.recv[f], self.peers[f]))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for f in self.faces:
            unpack(f, self.recv[f])


class SlabSolver:
    """An eu3d.Solver on this rank's x block of a (total_ni, nj, nk) grid.

    Every step first exchanges the halo planes with the neighbouring blocks,
    then runs the handle's step. Over NCCL the packs, the transfers and the
    unpacks are ordered on the handle's stream, with no host synchronisation;
    over a host backend (gloo) each message is staged through host memory.
    The ghost fill of the boundary condition applies only on the global
    domain's faces."""

    def __init__(self, dist, total_ni, total_nj, total_nk, extent, rank=None, ranks=None, device=0, **kw):
        import torch
        self.dist = dist
        self.rank = dist.get_rank() if rank is None else rank
        self.ranks = dist.get_world_size() if ranks is None else ranks
        self.first, self.n = block_range(total_ni, self.ranks, self.rank)
        self.total_ni = total_ni
        self.solver = eu3d.Solver(total_ni, total_nj, total_nk, extent, device=device, blocks_x=self.ranks,
                                  block_x=self.rank, **kw)
        self.device = torch.device("cuda", device)
        stream, _ = self.solver.device_info()
        self.stream = torch.cuda.ExternalStream(stream, device=self.device)
        self.halo = None
        self.dt_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.on_host = dist.get_backend() != "nccl"  # messages staged through host memory
        self.stage = {}

    # the handle's own calls (set_state, get, autotune, ...)
    def __getattr__(self, name):
        if name == "solver":
            raise AttributeError(name)
        return getattr(self.solver, name)

    def set_mechanism(self, m):
        import torch
        self.solver.set_mechanism(m)
        dtype = torch.float32 if self.solver.cfg.precision == eu3d.PRECISION["mixed"] else torch.float64
        numel = self.solver.halo_bytes() // (4 if dtype == torch.float32 else 8)
        self.halo = HaloExchange(self.dist, self.rank, self.ranks, numel, dtype,
                                 "cpu" if self.on_host else self.device)
        if self.on_host:
            self.stage = {f: torch.empty(numel, dtype=dtype, device=self.device) for f in self.halo.faces}

    def _pack(self, f, t):
        if not self.on_host:
            self.solver.halo_pack(f, t.data_ptr())
            return
        self.solver.halo_pack(f, self.stage[f].data_ptr())
        t.copy_(self.stage[f])  # synchronous: the message is on the host before it is sent

    def _unpack(self, f, t):
        if not self.on_host:
            self.solver.halo_unpack(f, t.data_ptr())
            return
        self.stage[f].copy_(t)
        self.solver.halo_unpack(f, self.stage[f].data_ptr())

    def exchange(self):
        import torch
        with torch.cuda.stream(self.stream):
            self.halo.exchange(self._pack, self._unpack)

    def _min_over_blocks(self, t):
        if not self.on_host:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
            return
        h = t.cpu()
        self.dist.all_reduce(h, op=self.dist.ReduceOp.MIN)
        t.copy_(h)

    def step(self, nsteps, dt, stats=True):
        """nsteps steps of fixed dt; stats of the last step (it synchronises)."""
        out = None
        for n in range(nsteps):
            self.exchange()
            out = self.solver.step(1, dt, stats=stats and n == nsteps - 1)
        return out

    def step_cfl(self, nsteps, cfl):
        """nsteps steps, each of the global CFL dt (minimum over the blocks, on
        the device). Returns (stats of the last step, time advanced)."""
        import torch
        time = torch.zeros(1, dtype=torch.float64, device=self.device)
        out = None
        for n in range(nsteps):
            self.exchange()
            with torch.cuda.stream(self.stream):
                self.solver.cfl_dt(cfl, self.dt_buf.data_ptr())
                self._min_over_blocks(self.dt_buf)
                out = self.solver.step_dt_device(1, self.dt_buf.data_ptr(), stats=n == nsteps - 1)
                time += self.dt_buf
        with torch.cuda.stream(self.stream):
            t = float(time.item())
        return out, t

    def interior(self, a, bc=2):
        """This block's interior nodes of a haloed field (planes, ni, nj, nk)."""
        return a[..., bc:-bc, bc:-bc, bc:-bc]

    def close(self):
        self.solver.close()


def gather_x(dist, block_interior, total_ni, rank, ranks):
    """Rank 0 receives every block's interior nodes (host arrays (..., n, nj, nk)
    of equal shape, over a process group that moves CPU tensors, e.g. gloo) and
    returns the global (..., total_ni, nj, nk) array, each shared node taken
    from the block on its left; other ranks return None."""
    import torch
    t = torch.as_tensor(np.ascontiguousarray(block_interior))
    parts = [torch.empty_like(t) for _ in range(ranks)] if rank == 0 else None
    dist.gather(t, parts, dst=0)
    if rank != 0:
        return None
    out = np.empty(block_interior.shape[:-3] + (total_ni,) + block_interior.shape[-2:], dtype=block_interior.dtype)
    for r in range(ranks - 1, -1, -1):  # right to left: a shared node keeps the left block's copy
        first, n = block_range(total_ni, ranks, r)
        out[..., first:first + n, :, :] = parts[r].numpy()
    return out
