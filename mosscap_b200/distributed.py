"""Slab decomposition of one 2D or 3D problem over ranks (one GPU per rank).

The global grid is split along its slowest active axis (y in 2D, z in 3D)
into equal slabs, one per rank. Each rank advances its slab with the fused
kernels. By default (transport "library") the library itself fills the
ghost layers between slabs after every stage and forms every dt from the
global CFL minimum, with NCCL in the stream (``mc_set_slab_decomposition``).
The other transports do the same from Python: the faces between slabs are
MC_BC_USERFN faces whose ghost rows are filled by the boundary hook of the C
ABI (``mc_set_user_bc``, the counterpart of ``Simulation::user_bc``,
source/Simulation.hpp:55), which the library calls after every stage and
after ``mc_fill_bcs``: the hook sends this rank's first / last ``ng``
interior rows to the neighbours below / above and receives their rows into
its ghost rows (``torch.distributed`` point-to-point). The step's dt is the
global CFL minimum (an all-reduce MIN of the per-rank minima, exact because
a minimum does not depend on order), clamped to the output times as
``compute_dt`` does (source/Hydro.cpp:231-241). A slab run is therefore
bit-identical to the single-domain run.

The outer y faces keep the global problem's kinds; periodic outer faces are
exchanged between the last and the first rank. ``SlabSim.advance`` runs the
device-driven loop instead: the global CFL minimum is then an in-stream
all-reduce through the library's CFL reduce hook (``mc_set_cfl_reduce_hook``)
and no step waits for the host.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import replace
from typing import Optional

import numpy as np
import torch
import torch.distributed as dist

from . import capi
from .hydro import HydroSim
from .problems import Problem


class _CudaArray:
    """A raw device pointer exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def exchange_rows(q: torch.Tensor, ng: int, ny: int, rank: int, world: int, periodic: bool,
                  group=None, via_host: bool = False) -> None:
    """Fill the y ghost rows of a slab from its neighbours.

    q: [nvar, 1, ny + 2 ng, xc] (this rank's slab with ghosts). Rows
    [ng, 2 ng) go to the rank below (its top ghosts), rows [ny, ny + ng) to
    the rank above (its bottom ghosts). Ranks 0 and world-1 exchange with each
    other only if the outer faces are periodic; otherwise their outer ghost
    rows are left to the kernels' own boundary handling. via_host: the rows
    travel through host memory (for a process group whose backend moves
    host tensors, e.g. gloo)."""
    lo_send = q[:, 0, ng:2 * ng, :].contiguous()
    hi_send = q[:, 0, ny:ny + ng, :].contiguous()
    if via_host:
        lo_send, hi_send = lo_send.cpu(), hi_send.cpu()
    below = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    above = rank + 1 if rank < world - 1 else (0 if periodic else None)
    if world == 1:
        if periodic:
            q[:, 0, 0:ng, :] = hi_send
            q[:, 0, ny + ng:ny + 2 * ng, :] = lo_send
        return
    lo_recv = torch.empty_like(lo_send)
    hi_recv = torch.empty_like(hi_send)
    # Messages travelling down (a slab's first rows to the rank below) come
    # first, then messages travelling up. With two ranks "below" and "above"
    # are the same peer, and point-to-point messages between one pair match in
    # issue order (NCCL has no tags), so both sides must issue the down
    # exchange before the up exchange.
    down, up = 1, 2
    ops = []
    if below is not None:
        ops.append(dist.P2POp(dist.isend, lo_send, below, group, tag=down))
    if above is not None:
        ops.append(dist.P2POp(dist.irecv, hi_recv, above, group, tag=down))
    if above is not None:
        ops.append(dist.P2POp(dist.isend, hi_send, above, group, tag=up))
    if below is not None:
        ops.append(dist.P2POp(dist.irecv, lo_recv, below, group, tag=up))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    if below is not None:
        q[:, 0, 0:ng, :] = lo_recv.to(q.device)
    if above is not None:
        q[:, 0, ny + ng:ny + 2 * ng, :] = hi_recv.to(q.device)


def clamp_to_output(dt: float, time: float, max_time: float, prev_output_time: float, delta: float) -> float:
    """The output-time clamp of compute_dt (source/Hydro.cpp:231-241)."""
    cand = prev_output_time + delta
    next_write = cand if cand < max_time else max_time
    if time + dt >= next_write:
        dt = next_write - time
        while time + dt < next_write:
            dt = math.nextafter(dt, math.inf)
    return dt


class SlabSim:
    """This rank's slab of a 2D (3D) problem split along y (z) over `world` ranks."""

    def __init__(self, problem: Problem, rank: int = 0, world: int = 1, precision: str = "fp64",
                 device: Optional[torch.device] = None, group=None, is_slab: bool = False,
                 transport: str = "library"):
        """problem: the global problem, whose rows (2D) or planes (3D) are
        split over the ranks; or, with is_slab, this rank's slab itself (its
        rows or planes and their ghost layers, the global problem's face
        kinds), so that no rank builds the global state.

        transport: "library" -- the library fills the ghost layers between
        slabs after every stage and reduces the CFL minimum over the ranks
        itself, with NCCL in the stream (mc_set_slab_decomposition; 2D and
        3D); "hook" -- this module fills them through the boundary hook and
        reduces through the CFL reduce hook with torch.distributed on device
        tensors (2D); "host" -- the same staged through host memory, for a
        gloo process group (2D)."""
        p = problem
        if p.num_dim not in (2, 3) or transport not in ("library", "hook", "host"):
            raise ValueError("a 2D or 3D problem and a known transport")
        if p.num_dim == 3 and transport != "library":
            raise ValueError("3D slabs use the library transport")
        self.axis = p.num_dim - 1
        n_glob = p.ny if self.axis == 1 else p.nz
        if not is_slab and n_glob % world != 0:
            raise ValueError("the slab axis's cell count must divide by the number of ranks")
        self.rank, self.world, self.group = rank, world, group
        self.transport = transport
        self.via_host = transport == "host"
        self.ng = p.ng
        self.n = n_glob if is_slab else n_glob // world
        self.ny = self.n  # rows per slab (2D)
        fa = 2 * self.axis
        self.periodic_y = p.bc[fa] == "periodic"
        bc = list(p.bc)
        if transport != "library":
            if rank > 0 or self.periodic_y:
                bc[fa] = "userfn"
            if rank < world - 1 or self.periodic_y:
                bc[fa + 1] = "userfn"
        ng = p.ng
        if is_slab:
            local = replace(p, bc=tuple(bc))
        elif self.axis == 1:
            rows = slice(rank * self.n, rank * self.n + self.n + 2 * ng)
            local = replace(p, ny=self.n, bc=tuple(bc),
                            loc=(p.loc[0], p.loc[1] + rank * self.n * p.dx, p.loc[2]),
                            Q=np.ascontiguousarray(p.Q[:, :, rows, :]))
        else:
            planes = slice(rank * self.n, rank * self.n + self.n + 2 * ng)
            local = replace(p, nz=self.n, bc=tuple(bc),
                            loc=(p.loc[0], p.loc[1], p.loc[2] + rank * self.n * p.dx),
                            Q=np.ascontiguousarray(p.Q[:, planes, :, :]))
        self.problem = local
        self.sim = HydroSim(local, precision=precision, device=device)
        self._fused_min_valid = False
        lib = self.sim.lib
        if transport == "library":
            uid = ctypes.create_string_buffer(128)
            if rank == 0:
                capi.check(lib.mc_slab_unique_id(uid), "mc_slab_unique_id")
            if world > 1:
                box = [uid.raw]
                dist.broadcast_object_list(box, src=0, group=group)
                uid = ctypes.create_string_buffer(box[0], 128)
            capi.check(lib.mc_set_slab_decomposition(self.sim.ctx, uid, rank, world), "mc_set_slab_decomposition")
            return
        self._hook = capi.USER_BC_FN(self._fill_rows)
        capi.check(lib.mc_set_user_bc(self.sim.ctx, self._hook, None), "mc_set_user_bc")
        # the domain-wide CFL minimum of the device-driven loop: an in-stream
        # all-reduce MIN of the 64-bit word holding the bits of the
        # non-negative minimum (integer order = value order)
        self._reduce = capi.CFL_REDUCE_FN(self._reduce_min)
        if world > 1:
            capi.check(lib.mc_set_cfl_reduce_hook(self.sim.ctx, self._reduce, None), "mc_set_cfl_reduce_hook")

    def _reduce_min(self, user, ptr, stream):
        word = torch.as_tensor(_CudaArray(ptr, (1,), "<i8"), device=self.sim.device)
        if self.via_host:
            h = word.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.MIN, group=self.group)
            word.copy_(h)
        else:
            dist.all_reduce(word, op=dist.ReduceOp.MIN, group=self.group)

    def _fill_rows(self, user, qptr, stream):
        shape = tuple(self.sim.Q.shape)
        q = torch.as_tensor(_CudaArray(qptr, shape), device=self.sim.device)
        exchange_rows(q, self.ng, self.ny, self.rank, self.world, self.periodic_y, self.group, self.via_host)

    @property
    def time(self) -> float:
        return self.sim.time

    def fill_bcs(self) -> None:
        self.sim.fill_bcs()
        self._fused_min_valid = False

    def compute_dt(self) -> float:
        """Global dt. With the library transport mc_compute_dt reduces over
        the ranks itself. Otherwise, after a step the local minimum is the one
        the step's last stage reduced (interior and in-plane ghosts; the
        exchanged ghost layers hold neighbours' cells, which the neighbours
        count), so no extra pass."""
        if self.transport == "library":
            return self.sim.compute_dt()
        if self._fused_min_valid:
            local = self.sim.last_cfl_min() * self.sim.problem.max_cfl
        else:
            local = self.sim.compute_dt(clamp=False)
        if self.world > 1:
            t = torch.tensor([local], dtype=torch.float64, device="cpu" if self.via_host else self.sim.device)
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
            local = float(t.item())
        s = self.sim
        return clamp_to_output(local, s.time, s.max_time, s.prev_output_time, s.output_delta)

    def advance(self, max_steps: int):
        """Up to max_steps steps in the device-driven loop (mc_advance): ghost
        layers exchanged after every stage, the global CFL minimum formed
        before every dt, in the stream; no host round trip per step. Returns
        the dt of each step."""
        self._fused_min_valid = False
        return self.sim.advance(max_steps)

    def step(self) -> float:
        dt = self.compute_dt()
        self.sim.time_step(dt)
        self._fused_min_valid = True
        s = self.sim
        if s.time >= s.prev_output_time + s.output_delta:
            s.prev_output_time = s.time
        return dt

    def interior(self) -> np.ndarray:
        ng = self.ng
        q = self.sim.get_Q()
        if self.axis == 1:
            return q[:, :, ng:-ng, ng:-ng]
        return q[:, ng:-ng, ng:-ng, ng:-ng]


def partition_by_cost(costs, world: int):
    """Split independent problems over `world` ranks by cost (for a batch:
    interior cells, every problem taking the same number of steps): largest
    first, each to the rank with the least load so far (the greedy
    longest-processing-time rule; its largest load is within 4/3 of the
    optimum). Returns one list of problem indices per rank, each in
    ascending order. The problems need no exchange, so the ranks share
    nothing but the timing."""
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(k)
        loads[r] += costs[k]
    return [sorted(p) for p in parts]
