"""The x decomposition on one GPU: two or three block handles of one grid
(cfg.blocks_x) in one process, their halo messages moved through device buffers
between the steps (the transfer NCCL makes between ranks), against the C
restatement's blocks and against the grid run as one block.

Blocks share a node and extrapolate their own ghost coordinates (Mesh::Boundary,
src/Mesh.cpp:131-142), so near a shared node a block may differ from the
one-block run by rounding; beyond the nodes an interface reaches in the steps
taken (two per step, plus the stencil) they are bitwise equal."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from helpers import golden_mechanism, rel_linf

sys.path.insert(0, os.path.join(ROOT, "eu3d-gpu_b200"))
import eu3d_cases as cases  # noqa: E402
import slab  # noqa: E402

pytestmark = pytest.mark.gpu

NI, NJ, NK = 61, 17, 19
EXT = (0.0, 0.060, 0.0, 0.016, 0.0, 0.018)


def _prim(mech, x, y, z):
    return cases.shock_bubble(x, y, z, mech["mw"], mech["ns"], radius=5e-3, shock_x=16e-3, standoff=8e-3, seed=3)


def _mech_dict(m):
    return {k: getattr(m, k) for k in ("ns", "nr", "mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f",
                                       "stoi_b", "tb")}


def _global_prim(mech):
    x = cases.node_coordinates(NI, EXT[0], EXT[1])
    y = cases.node_coordinates(NJ, EXT[2], EXT[3])
    z = cases.node_coordinates(NK, EXT[4], EXT[5])
    return (x, y, z), _prim(mech, x, y, z)


def _blocks(gpu, mech, prim, blocks, **kw):
    out = []
    for b in range(blocks):
        s = gpu.Solver(NI, NJ, NK, EXT, blocks_x=blocks, block_x=b, **kw)
        s.set_mechanism(mech)
        s.set_primitive(*[slab.block_slice(np.asarray(a), NI, blocks, b) for a in prim])
        out.append(s)
    return out


def _exchange(blocks, bufs):
    """One step's halo transfer between the block handles (host-ordered)."""
    for s in blocks:
        s.sync()
    for r, s in enumerate(blocks):
        if r > 0:
            s.halo_pack(0, bufs[r][0].data_ptr())
        if r < len(blocks) - 1:
            s.halo_pack(1, bufs[r][1].data_ptr())
    for s in blocks:
        s.sync()
    for r, s in enumerate(blocks):
        if r > 0:
            s.halo_unpack(0, bufs[r - 1][1].data_ptr())
        if r < len(blocks) - 1:
            s.halo_unpack(1, bufs[r + 1][0].data_ptr())


def _buffers(blocks):
    import torch
    n = blocks[0].halo_bytes()
    return [[torch.empty(n, dtype=torch.uint8, device="cuda:0") for _ in range(2)] for _ in blocks]


def _gather(blocks, name):
    parts = [s.get(name)[:, 2:-2, 2:-2, 2:-2] for s in blocks]
    out = np.empty(parts[0].shape[:1] + (NI,) + parts[0].shape[2:])
    for r in range(len(blocks) - 1, -1, -1):
        first, n = slab.block_range(NI, len(blocks), r)
        out[:, first:first + n] = parts[r]
    return out


def _far(blocks, steps):
    reach = 2 * steps + 3
    far = np.ones(NI, bool)
    for r in range(1, blocks):
        s = slab.block_range(NI, blocks, r)[0]
        far[max(s - reach, 0):s + reach + 1] = False
    assert far.any()
    return far


def test_block_nodes_follow_the_reference_layout(gpu):
    """Mesh::Initial's node positions (global spacing, block offset) and
    Mesh::Boundary's extrapolated ghosts, per block."""
    mech = _mech_dict(golden_mechanism())
    (xg, _, _), prim = _global_prim(mech)
    blocks = _blocks(gpu, mech, prim, 3)
    for r, s in enumerate(blocks):
        first, n = slab.block_range(NI, 3, r)
        x = s.nodes()[0]
        assert len(x) == n + 4
        assert np.array_equal(x[2:-2], xg[2 + first:2 + first + n])
        assert np.array_equal(x, cases.node_coordinates(NI, EXT[0], EXT[1], blocks=3, block=r))
        s.close()


def test_halo_messages_carry_the_neighbours_nodes(gpu):
    """Face 1 of a block packs the two nodes left of its last one; face 0 of
    the next block unpacks them into its ghost planes 1 and 0 (and the other
    way round), as Flowfield::Mpi_Boundary moves them."""
    import torch
    mech = _mech_dict(golden_mechanism())
    _, prim = _global_prim(mech)
    a, b = _blocks(gpu, mech, prim, 2)
    bufs = _buffers([a, b])
    _exchange([a, b], bufs)
    a.sync()
    b.sync()
    pa, pb = a.get("P"), b.get("P")
    n = slab.block_range(NI, 2, 0)[1]
    # shared node: a's last interior node (n + 1) is b's first (2)
    assert np.array_equal(pb[0, 1], pa[0, n]) and np.array_equal(pb[0, 0], pa[0, n - 1])
    assert np.array_equal(pa[0, n + 2], pb[0, 3]) and np.array_equal(pa[0, n + 3], pb[0, 4])
    msg = bufs[0][1].view(torch.float64).cpu().numpy().reshape(16, 2, NJ + 4, NK + 4)
    assert np.array_equal(msg[0, 0], pa[0, n]) and np.array_equal(msg[0, 1], pa[0, n - 1])
    a.close()
    b.close()


@pytest.mark.parametrize("blocks", [2, 3])
def test_blocks_match_restatement_blocks_and_one_block(gpu, port_lib, blocks):
    """FP64 strict stiff steps: the GPU blocks against the C restatement's
    blocks (same decomposition, messages copied between them) to the usual
    restatement tolerance, and against the one-block GPU run bitwise away from
    the shared nodes."""
    import oracle
    steps, dt = 6, 5e-8
    mech_o = golden_mechanism()
    mech = _mech_dict(mech_o)
    (x, y, z), prim = _global_prim(mech)
    gblocks = _blocks(gpu, mech, prim, blocks, record_sources=True)
    bufs = _buffers(gblocks)
    ports = []
    for r in range(blocks):
        first, n = slab.block_range(NI, blocks, r)
        p = port_lib(n, NJ, NK, cases.node_coordinates(NI, EXT[0], EXT[1], blocks=blocks, block=r), y, z, mech_o)
        p.set_primitive(*[slab.block_slice(np.asarray(a), NI, blocks, r) for a in prim])
        p.set_exchange(r > 0, r < blocks - 1)
        ports.append(p)
    msgs = [[np.empty(ports[0].halo_count()) for _ in range(2)] for _ in ports]
    for _ in range(steps):
        _exchange(gblocks, bufs)
        for s in gblocks:
            s.step(1, dt, stats=False)
        for r, p in enumerate(ports):
            if r > 0:
                p.halo_pack(0, msgs[r][0])
            if r < blocks - 1:
                p.halo_pack(1, msgs[r][1])
        for r, p in enumerate(ports):
            if r > 0:
                p.halo_unpack(0, msgs[r - 1][1])
            if r < blocks - 1:
                p.halo_unpack(1, msgs[r + 1][0])
            p.step(1, dt)
    one = gpu.Solver(NI, NJ, NK, EXT, record_sources=True)
    one.set_mechanism(mech)
    one.set_primitive(*prim)
    one.step(steps, dt)
    far = _far(blocks, steps)
    for name in ("CS", "T", "Yi"):
        got = _gather(gblocks, name)
        port = np.empty_like(got)
        for r in range(blocks - 1, -1, -1):
            first, n = slab.block_range(NI, blocks, r)
            port[:, first:first + n] = ports[r].get(name)[:, 2:-2, 2:-2, 2:-2]
        assert rel_linf(got, port).max() <= 1e-10, name
        ref = one.get(name)[:, 2:-2, 2:-2, 2:-2]
        assert rel_linf(got, ref).max() <= 1e-12, name
        assert np.array_equal(got[:, far], ref[:, far]), name
    for s in gblocks + [one]:
        s.close()


def test_mixed_learned_blocks_match_one_block(gpu):
    """The learned + mixed step (FP32 messages) in three blocks against one
    block: bitwise away from the shared nodes, within FP32 rounding near them."""
    import learned
    steps = 5
    mech = _mech_dict(golden_mechanism())
    (x, y, z), prim = _global_prim(mech)
    model, gate = learned.load(device=0)
    kw = dict(precision="mixed", chemistry="learned", arith="fast")
    gblocks = _blocks(gpu, mech, prim, 3, **kw)
    for s in gblocks:
        learned.attach(s, model, gate)
    one = gpu.Solver(NI, NJ, NK, EXT, **kw)
    one.set_mechanism(mech)
    one.set_primitive(*prim)
    learned.attach(one, model, gate)
    D = one.get("D")
    P = one.get("P")
    dt = cases.cfl_dt(x, y, P[0], D[0], one.get("U")[0], one.get("V")[0], one.get("Gamma")[0], 0.5)
    bufs = _buffers(gblocks)
    assert gblocks[0].halo_bytes() == 16 * 2 * (NJ + 4) * (NK + 4) * 4
    for _ in range(steps):
        _exchange(gblocks, bufs)
        for s in gblocks:
            s.step(1, dt, stats=False)
    one.step(steps, dt)
    far = _far(3, steps)
    for name in ("CS", "T"):
        got = _gather(gblocks, name)
        ref = one.get(name)[:, 2:-2, 2:-2, 2:-2]
        assert rel_linf(got, ref).max() <= 1e-6, name
        assert np.array_equal(got[:, far], ref[:, far]), name
    for s in gblocks + [one]:
        s.close()


def test_cfl_dt_on_the_device_matches_step_cfl(gpu):
    """eu_cfl_dt + eu_step_dt_device (the split the blocks use, with the
    minimum over blocks in between) step exactly as eu_step_cfl."""
    import torch
    mech = _mech_dict(golden_mechanism())
    _, prim = _global_prim(mech)
    a = gpu.Solver(NI, NJ, NK, EXT, precision="mixed", arith="fast")
    b = gpu.Solver(NI, NJ, NK, EXT, precision="mixed", arith="fast")
    for s in (a, b):
        s.set_mechanism(mech)
        s.set_primitive(*prim)
    _, t = a.step_cfl(4, 0.5)
    dt = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    total = 0.0
    for _ in range(4):
        b.cfl_dt(0.5, dt.data_ptr())
        b.step_dt_device(1, dt.data_ptr())
        b.sync()
        total += float(dt.item())
    assert total == t
    for name in ("CS", "T"):
        assert np.array_equal(a.get(name), b.get(name)), name
    a.close()
    b.close()


def _slab_rank(rank, ranks, port, out):
    """One rank of the two-process run: a SlabSolver over a gloo group on
    cuda:0 (messages staged through host memory)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "eu3d-gpu_b200"),
                    os.path.join(ROOT, "tests")]
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    import learned
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ranks, timeout=timedelta(seconds=120))
    mech = _mech_dict(golden_mechanism())
    _, prim = _global_prim(mech)
    s = slab.SlabSolver(dist, NI, NJ, NK, EXT, device=0, precision="mixed", chemistry="learned", arith="fast")
    s.set_mechanism(mech)
    s.set_primitive(*[slab.block_slice(np.asarray(a), NI, ranks, rank) for a in prim])
    model, gate = learned.load(device=0)
    learned.attach(s.solver, model, gate)
    s.step(4, 4e-8)
    fixed = {n: slab.gather_x(dist, s.get(n)[:, 2:-2, 2:-2, 2:-2], NI, rank, ranks) for n in ("CS", "T")}
    _, t = s.step_cfl(2, 0.5)
    after = slab.gather_x(dist, s.get("CS")[:, 2:-2, 2:-2, 2:-2], NI, rank, ranks)
    s.close()
    dist.destroy_process_group()
    if rank == 0:
        out.put((fixed, t, after))


def test_slab_solver_in_two_processes_matches_one_block(gpu):
    """eu3d-gpu_b200/slab.py's SlabSolver as two ranks (gloo, both on this GPU,
    host-staged messages; their kernels never wait on each other): four
    fixed-dt steps bitwise equal to one block away from the shared node, then
    two steps with the CFL dt reduced over the blocks."""
    import socket
    import torch.multiprocessing as mp
    import learned
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_slab_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    fixed, t, after = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]

    mech = _mech_dict(golden_mechanism())
    _, prim = _global_prim(mech)
    one = gpu.Solver(NI, NJ, NK, EXT, precision="mixed", chemistry="learned", arith="fast")
    one.set_mechanism(mech)
    one.set_primitive(*prim)
    model, gate = learned.load(device=0)
    learned.attach(one, model, gate)
    one.step(4, 4e-8)
    far = _far(2, 4)
    for n in ("CS", "T"):
        ref = one.get(n)[:, 2:-2, 2:-2, 2:-2]
        assert rel_linf(fixed[n], ref).max() <= 1e-6, n
        assert np.array_equal(fixed[n][:, far], ref[:, far]), n
    _, t_one = one.step_cfl(2, 0.5)
    assert abs(t - t_one) <= 1e-9 * t_one
    assert rel_linf(after, one.get("CS")[:, 2:-2, 2:-2, 2:-2]).max() <= 1e-5
    one.close()


def _bench_rank(rank, ranks, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "eu3d-gpu_b200")]
    import argparse
    import contextlib
    import io
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    import bench
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ranks, timeout=timedelta(seconds=300))
    args = argparse.Namespace(grid=[33, 17, 17], chem="learned", precision="mixed", arith="fast", steps=2, warmup=3,
                              no_autotune=False, window_start=5, total_steps=12)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = bench.our_arm_blocks(args, ranks, rank, 0, dist)
    out.put((rank, rc, buf.getvalue()))


def test_bench_block_arm_in_two_processes(gpu):
    """bench.py's decomposed arm (the one `--gpus N` runs under torchrun) as
    two gloo ranks on this GPU on a small grid: it finishes and rank 0 prints
    one JSON line with the global grid and the exchange in its config."""
    import json
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bench_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert [g[1] for g in got] == [0, 0]
    assert got[1][2] == ""
    line = json.loads(got[0][2].strip().splitlines()[-1])
    assert line["n_gpus"] == 2 and line["scaling"] == "weak" and line["value"] > 0
    assert line["config"]["global_grid"] == [65, 17, 17]
    assert "halo exchange" in line["config"]["parallelism"]
    assert line["e2e"]["value"] > 0 and line["gpu_launches"] > 0
