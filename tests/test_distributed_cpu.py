"""Multi-rank host logic of the slab decomposition on CPU: two (and three)
gloo ranks exchange ghost rows of their slabs; every ghost row must equal the
neighbouring slab's interior row of the global array (periodic or not)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, periodic, errors):
    from mosscap_b200.distributed import exchange_rows
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ng, ny, nx, nvar = 3, 5, 7, 4
        rng = np.random.default_rng(0)
        glob = rng.standard_normal((nvar, 1, world * ny, nx + 2 * ng))
        # global rows with periodic ghost rows
        pad = np.concatenate([glob[:, :, -ng:], glob, glob[:, :, :ng]], axis=2)
        mine = pad[:, :, rank * ny: rank * ny + ny + 2 * ng].copy()
        q = torch.from_numpy(mine.copy())
        q[:, 0, :ng] = -1.0
        q[:, 0, ny + ng:] = -1.0
        exchange_rows(q, ng, ny, rank, world, periodic)
        got = q.numpy()
        exp = mine.copy()
        if not periodic and rank == 0:
            exp[:, 0, :ng] = -1.0
        if not periodic and rank == world - 1:
            exp[:, 0, ny + ng:] = -1.0
        if not np.array_equal(got, exp):
            errors.put(f"rank {rank}: ghost rows differ")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic", [True, False])
def test_exchange_rows_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic, errors)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert errors.empty(), errors.get()


def test_clamp_to_output_matches_reference_rule():
    from mosscap_b200.distributed import clamp_to_output
    # no clamp
    assert clamp_to_output(0.01, 0.0, 1.0, 0.0, 0.1) == 0.01
    # clamped to the next output time, time + dt lands exactly on it
    t = 0.0949999
    dt = clamp_to_output(0.01, t, 1.0, 0.0, 0.1)
    # dt starts at next_write - time and only moves up until time + dt lands
    assert t + dt >= 0.1 and dt >= 0.1 - t and dt - (0.1 - t) < 1e-17
    # clamped to max_time
    dt = clamp_to_output(0.5, 0.9, 1.0, 0.0, 5.0)
    assert 0.9 + dt >= 1.0


def _min_worker(rank, world, port, errors):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(7)
        vals = np.concatenate([rng.uniform(0.0, 1e-3, size=(world, 64)), np.zeros((world, 1)),
                               np.full((world, 1), np.inf), 10.0 ** rng.uniform(-300, 300, size=(world, 64))], axis=1)
        mine = vals[rank]
        # what the CFL reduce hook of SlabSim does to the library's word: an
        # integer MIN over the bit patterns of the non-negative minima
        word = torch.from_numpy(mine.view(np.int64).copy())
        dist.all_reduce(word, op=dist.ReduceOp.MIN)
        got = word.numpy().view(np.float64)
        if not np.array_equal(got, vals.min(axis=0)):
            errors.put(f"rank {rank}: integer MIN of the bits is not the minimum")
    finally:
        dist.destroy_process_group()


def test_cfl_minimum_by_integer_min_of_bits():
    """The slab decomposition's global CFL minimum is an all-reduce MIN of
    the 64-bit words holding the bits of each rank's non-negative minimum
    (zero and +inf included): integer order equals value order."""
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_min_worker, args=(r, 3, port, errors)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert errors.empty(), errors.get()


@pytest.mark.parametrize("world", [2, 3, 8])
def test_partition_by_cost_balances_the_batch(world):
    """The seeded 4096-problem batch split over ranks by interior cells:
    every problem on exactly one rank, and the largest load within the
    greedy rule's bound (mean load plus the largest problem)."""
    from mosscap_b200 import problems as P
    from mosscap_b200.distributed import partition_by_cost
    probs = P.riemann_batch(seed=0, n1d=256, n2d=256)
    costs = [p.interior_cells for p in probs]
    parts = partition_by_cost(costs, world)
    flat = sorted(k for part in parts for k in part)
    assert flat == list(range(len(probs)))
    loads = [sum(costs[k] for k in part) for part in parts]
    assert max(loads) <= sum(costs) / world + max(costs)
    assert max(loads) / (sum(costs) / world) < 1.02


def _comm_worker(rank, world, port, errors):
    from mosscap_b200 import capi
    from mosscap_b200.adjoint import comm_op
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        count = 6
        # rank r sends its first rows (send_lo) down and its last rows up
        send_lo = torch.full((count,), 100.0 * rank + 1, dtype=torch.float64)
        send_hi = torch.full((count,), 100.0 * rank + 2, dtype=torch.float64)
        recv_lo = torch.zeros(count, dtype=torch.float64)
        recv_hi = torch.zeros(count, dtype=torch.float64)
        comm_op(capi.COMM_HALO, (send_lo, send_hi, recv_lo, recv_hi), rank, world, via_host=True)
        below, above = (rank - 1) % world, (rank + 1) % world
        # from below: its last rows; from above: its first rows
        if not torch.all(recv_lo == 100.0 * below + 2) or not torch.all(recv_hi == 100.0 * above + 1):
            errors.put(f"rank {rank}: halo {recv_lo[0].item()} {recv_hi[0].item()}")
        key = torch.tensor([0x7FFFFFFFFFFFFFFF if rank == 0 else (rank << 32) | (7 - rank)], dtype=torch.int64)
        comm_op(capi.COMM_MIN_I64, (key,), rank, world, via_host=True)
        if key.item() != ((1 << 32) | 6):
            errors.put(f"rank {rank}: arg-min key {key.item():#x}")
        s = torch.tensor([0.5 * (rank + 1)], dtype=torch.float64)
        comm_op(capi.COMM_SUM_F64, (s,), rank, world, via_host=True)
        if s.item() != 0.25 * world * (world + 1):
            errors.put(f"rank {rank}: sum {s.item()}")
        bits = torch.tensor([np.float64(1.0 + rank).view(np.int64)], dtype=torch.int64)
        comm_op(capi.COMM_MIN_U64, (bits,), rank, world, via_host=True)
        if np.int64(bits.item()).view(np.float64) != 1.0:
            errors.put(f"rank {rank}: min {bits.item()}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_adjoint_slab_comm_hook_gloo(world):
    """The adjoint's slab hook operations (adjoint.comm_op) between gloo
    ranks: halo blocks travel to the ring neighbours (periodic, y order), the
    arg-min key reduces to the lowest rank holding a cell, sums and the
    double-bits minimum reduce in place."""
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_comm_worker, args=(r, world, port, errors)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert errors.empty(), errors.get()


def test_adjoint_slab_comm_hook_single_rank():
    """One rank is its own periodic neighbour; reductions are identities."""
    from mosscap_b200 import capi
    from mosscap_b200.adjoint import comm_op
    a, b = torch.arange(4.0, dtype=torch.float64), torch.arange(4.0, 8.0, dtype=torch.float64)
    lo, hi = torch.zeros(4, dtype=torch.float64), torch.zeros(4, dtype=torch.float64)
    comm_op(capi.COMM_HALO, (a, b, lo, hi), 0, 1)
    assert torch.equal(lo, b) and torch.equal(hi, a)
    s = torch.tensor([3.0], dtype=torch.float64)
    comm_op(capi.COMM_SUM_F64, (s,), 0, 1)
    assert s.item() == 3.0


def test_slab_adjoint_rejects_bad_partitions_on_the_host():
    """SlabAdjoint checks its partition before touching the device: the rows
    must divide by the ranks, the problem must be 2D and the transport known."""
    from mosscap_b200 import problems as P
    from mosscap_b200.adjoint import SlabAdjoint
    p = P.kelvin_helmholtz_2d(30, seed=0)
    with pytest.raises(ValueError):
        SlabAdjoint(p, p.gamma, rank=0, world=4)
    with pytest.raises(ValueError):
        SlabAdjoint(p, p.gamma, rank=0, world=2, transport="carrier-pigeon")
    with pytest.raises(ValueError):
        SlabAdjoint(P.sod_1d(64), 1.4)
