"""The x decomposition's host logic on the CPU: ranks as gloo processes, each
advancing its x block with the C restatement (oracle/eu3d_oracle.c) and moving
its halo messages with eu3d-gpu_b200/slab.py's HaloExchange, the code the GPU
ranks run over NCCL. The gathered blocks are compared with the same case run
as one block.

Neighbouring blocks share a node, and each block's ghost coordinates at an
internal face are extrapolated from its own nodes (Mesh::Boundary,
src/Mesh.cpp:131-142), so the spacing its first node's flux difference uses can
differ from the global grid's in the last bit. The reference's MPI runs carry
the same difference. The blocks therefore agree with the single-block run to
rounding near a shared node, and bitwise beyond the nodes an interface can
reach in the steps taken (two nodes per step, plus the stencil)."""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT
from helpers import golden_mechanism, rel_linf

sys.path.insert(0, os.path.join(ROOT, "eu3d-gpu_b200"))
import eu3d_cases as cases  # noqa: E402
import slab  # noqa: E402

NI, NJ, NK = 61, 9, 9
EXT = (0.0, 0.060, 0.0, 0.008, 0.0, 0.008)
STEPS, DT = 4, 1e-7


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(boundary, blocks=1, block=0):
    """Coordinates and primitive fields of one block (the whole grid when blocks
    == 1), and the ODW inflow tables (None for the other cases)."""
    mech = golden_mechanism()
    x = cases.node_coordinates(NI, EXT[0], EXT[1], blocks=blocks, block=block)
    xg = cases.node_coordinates(NI, EXT[0], EXT[1])
    y = cases.node_coordinates(NJ, EXT[2], EXT[3])
    z = cases.node_coordinates(NK, EXT[4], EXT[5])
    inflow = None
    if boundary == "znd":
        prim = cases.znd(xg, y, z, mech.mw, mech.ns)
    elif boundary == "odw":
        md = {k: getattr(mech, k) for k in ("ns", "mw", "coeff_lo", "coeff_hi")}
        prim, inflow = cases.odw(xg, y, z, md)
    else:
        prim = cases.shock_bubble(xg, y, z, mech.mw, mech.ns, radius=4e-3, shock_x=16e-3, standoff=6e-3, seed=3)
    if blocks > 1:  # the block's planes of the global fields
        prim = [slab.block_slice(np.asarray(a), NI, blocks, block) for a in prim]
    return mech, x, y, z, prim, inflow


def _run_block(rank, ranks, port, boundary, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "eu3d-gpu_b200"),
                    os.path.join(ROOT, "tests")]
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    import oracle
    dist.init_process_group("gloo", rank=rank, world_size=ranks, timeout=timedelta(seconds=60))
    mech, x, y, z, prim, inflow = _case(boundary, ranks, rank)
    first, n = slab.block_range(NI, ranks, rank)
    port_ = oracle.PortOracle(n, NJ, NK, x, y, z, mech, nthreads=1, boundary=boundary)
    port_.set_primitive(*prim)
    if inflow is not None:  # every block holds the tables; only the x-low one fills from them
        port_.set_inflow(*inflow)
    port_.set_exchange(rank > 0, rank < ranks - 1)
    halo = slab.HaloExchange(dist, rank, ranks, port_.halo_count(), torch.float64, "cpu")
    for _ in range(STEPS):
        halo.exchange(lambda f, t: port_.halo_pack(f, t.numpy()), lambda f, t: port_.halo_unpack(f, t.numpy()))
        port_.step(1, DT)
    fields = {name: slab.gather_x(dist, port_.get(name)[:, 2:-2, 2:-2, 2:-2], NI, rank, ranks)
              for name in ("CS", "T", "Yi")}
    dist.destroy_process_group()
    if rank == 0:
        out.put(fields)


@pytest.mark.parametrize("boundary,ranks", [("rsbi", 3), ("znd", 2), ("odw", 2)])
def test_blocks_match_one_block(port_lib, boundary, ranks):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run_block, args=(r, ranks, port, boundary, q)) for r in range(ranks)]
    for p in procs:
        p.start()
    got = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]

    mech, x, y, z, prim, inflow = _case(boundary)
    one = port_lib(NI, NJ, NK, x, y, z, mech, boundary=boundary)
    one.set_primitive(*prim)
    if inflow is not None:
        one.set_inflow(*inflow)
    one.step(STEPS, DT)
    reach = 2 * STEPS + 3
    shared = [slab.block_range(NI, ranks, r)[0] for r in range(1, ranks)]
    far = np.ones(NI, bool)
    for s in shared:
        far[max(s - reach, 0):s + reach + 1] = False
    assert far.any()
    for name in ("CS", "T", "Yi"):
        ref = one.get(name)[:, 2:-2, 2:-2, 2:-2]
        assert rel_linf(got[name], ref).max() <= 1e-12, name
        assert np.array_equal(got[name][:, far], ref[:, far]), name
