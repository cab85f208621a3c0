"""Differentiable Euler steps: a thin ``torch.autograd.Function`` over the
discrete adjoint of the C ABI (``mc_adjoint_*``).

``EulerSteps.apply(q0, gamma, problem, n_steps, checkpoint_every)`` maps the
interior conserved state ``q0`` (float64 CUDA tensor ``[4, ny, nx]``) and the
scalar ``gamma`` to the interior state after ``n_steps`` SSPRK3 steps of the
2D WENO5-Z + HLLC scheme with periodic faces. The forward pass runs the
fused FP64 kernels (ghost cells filled periodically from ``q0``); the
backward pass runs ``mc_adjoint_backward``, i.e. the exact vector-Jacobian
product of the discrete map, including each step's CFL dt and gamma.

``SlabAdjoint`` runs the same adjoint split into y slabs over ranks
(``mc_adjoint_set_slab_decomposition`` / ``mc_adjoint_set_slab_hook``).

``kh_initial_state(vy, gamma, problem)`` builds the Kelvin-Helmholtz initial
state from a perturbation field ``vy`` in torch operations (the same
``prim_to_cons`` as the reference), so that gradients with respect to the
initial ``vy`` field and ``gamma`` flow through the initial condition too.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch
import torch.distributed as dist

from . import capi
from .distributed import _CudaArray
from .hydro import grid_of
from .problems import Problem


def _scheme(problem: Problem, gamma: float) -> capi.McScheme:
    s = capi.McScheme()
    s.reconstruction = capi.RECON[problem.reconstruction]
    s.slope_limiter = capi.LIMITER[problem.slope_limiter]
    s.riemann_solver = capi.RIEMANN[problem.riemann_solver]
    s.time_stepper = capi.STEPPER[problem.time_stepper]
    s.precision = capi.PRECISION["fp64"]
    s.gamma = float(gamma)
    s.max_cfl = problem.max_cfl
    return s


def pad_periodic(q: torch.Tensor, ng: int) -> torch.Tensor:
    """[v, ny, nx] -> [v, 1, ny + 2 ng, nx + 2 ng] with periodic ghosts."""
    q = torch.cat([q[:, -ng:, :], q, q[:, :ng, :]], dim=1)
    q = torch.cat([q[:, :, -ng:], q, q[:, :, :ng]], dim=2)
    return q.unsqueeze(1).contiguous()


class _Runner:
    """Owns one mc_adjoint for a (problem, gamma) pair."""

    def __init__(self, problem: Problem, gamma: float, checkpoint_every: int):
        self.lib = capi.load()
        self.problem = problem
        self.grid = grid_of(problem)
        self.scheme = _scheme(problem, gamma)
        h = ctypes.c_void_p()
        capi.check(self.lib.mc_adjoint_create(ctypes.byref(self.grid), ctypes.byref(self.scheme),
                                              int(checkpoint_every), ctypes.byref(h)), "mc_adjoint_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.mc_adjoint_destroy(self.h)
            self.h = None

    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def forward(self, qpad: torch.Tensor, n_steps: int) -> None:
        clk = capi.McClock()
        clk.time, clk.max_time = 0.0, 1e300
        clk.prev_output_time, clk.output_delta = 0.0, 1e300
        capi.check(self.lib.mc_adjoint_forward(self.h, ctypes.c_void_p(qpad.data_ptr()), ctypes.byref(clk),
                                               int(n_steps), self.stream()), "mc_adjoint_forward")

    def backward(self, lam: torch.Tensor) -> float:
        g = ctypes.c_double()
        capi.check(self.lib.mc_adjoint_backward(self.h, ctypes.c_void_p(lam.data_ptr()), ctypes.byref(g),
                                                self.stream()), "mc_adjoint_backward")
        return g.value


class EulerSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0: torch.Tensor, gamma: torch.Tensor, problem: Problem, n_steps: int,
                checkpoint_every: int = 20) -> torch.Tensor:
        ng = problem.ng
        runner = _Runner(problem, float(gamma), checkpoint_every)
        qpad = pad_periodic(q0.detach().to(torch.float64), ng)
        runner.forward(qpad, n_steps)
        ctx.runner = runner
        ctx.ng = ng
        return qpad[:, 0, ng:-ng, ng:-ng].clone()

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        ng = ctx.ng
        lam = pad_periodic(grad_out.contiguous().to(torch.float64), ng) * 0.0
        lam[:, 0, ng:-ng, ng:-ng] = grad_out
        dgamma = ctx.runner.backward(lam)
        grad_q0 = lam[:, 0, ng:-ng, ng:-ng].clone()
        return grad_q0, torch.tensor(dgamma, dtype=torch.float64, device=grad_out.device), None, None, None


def comm_op(op: int, bufs, rank: int, world: int, group=None, via_host: bool = False) -> None:
    """One call of the adjoint's slab hook on tensors (mc_comm_fn semantics):
    ``capi.COMM_HALO`` with bufs = (send_lo, send_hi, recv_lo, recv_hi), the
    ranks forming a periodic ring in y order (send_lo to rank - 1, which
    receives it in its recv_hi; send_hi to rank + 1, into its recv_lo); a
    reduction with bufs = (buf,), all-reduced in place (``COMM_MIN_U64`` on the
    int64 view of non-negative double bits, whose signed order is their
    unsigned order). via_host: the data travel through host memory (a process
    group whose backend moves host tensors, e.g. gloo)."""
    if op == capi.COMM_HALO:
        send_lo, send_hi, recv_lo, recv_hi = bufs
        if world == 1:
            recv_lo.copy_(send_hi)
            recv_hi.copy_(send_lo)
            return
        below, above = (rank - 1) % world, (rank + 1) % world
        if via_host:
            s_lo, s_hi = send_lo.cpu(), send_hi.cpu()
            r_lo, r_hi = torch.empty_like(s_lo), torch.empty_like(s_hi)
        else:
            s_lo, s_hi, r_lo, r_hi = send_lo, send_hi, recv_lo, recv_hi
        # down (to the rank below) first, then up; with two ranks the two
        # neighbours are one peer and its messages match in issue order
        down, up = 1, 2
        ops = [dist.P2POp(dist.isend, s_lo, below, group, tag=down),
               dist.P2POp(dist.irecv, r_hi, above, group, tag=down),
               dist.P2POp(dist.isend, s_hi, above, group, tag=up),
               dist.P2POp(dist.irecv, r_lo, below, group, tag=up)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        if via_host:
            recv_lo.copy_(r_lo)
            recv_hi.copy_(r_hi)
        return
    (buf,) = bufs
    if world == 1:
        return
    red = dist.ReduceOp.SUM if op == capi.COMM_SUM_F64 else dist.ReduceOp.MIN
    if via_host:
        h = buf.cpu()
        dist.all_reduce(h, op=red, group=group)
        buf.copy_(h)
    else:
        dist.all_reduce(buf, op=red, group=group)


class SlabAdjoint:
    """This rank's y slab of the discrete adjoint of a periodic 2D problem
    split into ``world`` equal slabs, rank 0 holding the lowest rows.

    transport: "library" -- the library exchanges rows and reduces with NCCL
    in the stream (``mc_adjoint_set_slab_decomposition``); "hook" / "host" --
    through ``mc_adjoint_set_slab_hook`` with torch.distributed on device
    tensors / staged through host memory (gloo). The forward run is
    bit-identical to the single domain; the gradient differs from it only in
    the order of the dt and gamma sums over the ranks."""

    def __init__(self, problem: Problem, gamma: float, rank: int = 0, world: int = 1, checkpoint_every: int = 20,
                 transport: str = "library", group=None, device: Optional[torch.device] = None):
        if problem.num_dim != 2 or problem.ny % world != 0:
            raise ValueError("a 2D problem whose rows divide by the number of ranks")
        if transport not in ("library", "hook", "host"):
            raise ValueError("transport is library, hook or host")
        self.lib = capi.load()
        self.problem = problem
        self.rank, self.world, self.group = rank, world, group
        self.via_host = transport == "host"
        self.device = torch.device(device or "cuda")
        self.ng = problem.ng
        self.n = problem.ny // world
        self.grid = grid_of(problem)
        self.grid.yc = self.n + 2 * self.ng
        self.scheme = _scheme(problem, gamma)
        h = ctypes.c_void_p()
        capi.check(self.lib.mc_adjoint_create(ctypes.byref(self.grid), ctypes.byref(self.scheme),
                                              int(checkpoint_every), ctypes.byref(h)), "mc_adjoint_create")
        self.h = h
        self.hook_error = None
        if transport == "library":
            uid = ctypes.create_string_buffer(128)
            if rank == 0:
                capi.check(self.lib.mc_slab_unique_id(uid), "mc_slab_unique_id")
            if world > 1:
                box = [uid.raw]
                dist.broadcast_object_list(box, src=0, group=group)
                uid = ctypes.create_string_buffer(box[0], 128)
            capi.check(self.lib.mc_adjoint_set_slab_decomposition(self.h, uid, rank, world),
                       "mc_adjoint_set_slab_decomposition")
        else:
            self._hook = capi.COMM_FN(self._comm)
            capi.check(self.lib.mc_adjoint_set_slab_hook(self.h, self._hook, None, rank, world),
                       "mc_adjoint_set_slab_hook")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.mc_adjoint_destroy(self.h)
            self.h = None

    def _comm(self, user, op, bufs, count, stream):
        try:
            if op == capi.COMM_HALO:
                ts = [torch.as_tensor(_CudaArray(bufs[k], (count,)), device=self.device) for k in range(4)]
            else:
                typestr = "<f8" if op == capi.COMM_SUM_F64 else "<i8"
                ts = [torch.as_tensor(_CudaArray(bufs[0], (count,), typestr), device=self.device)]
            comm_op(op, ts, self.rank, self.world, self.group, self.via_host)
            return 0
        except Exception as e:  # reported by the library call as MC_ERR_CUDA
            self.hook_error = e
            return 1

    def _check(self, status, where):
        if status != capi.MC_OK and self.hook_error is not None:
            raise RuntimeError(f"{where}: slab hook failed") from self.hook_error
        capi.check(status, where)

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def rows(self, x: torch.Tensor) -> torch.Tensor:
        """This rank's rows of a global interior field [..., ny, nx]."""
        return x[..., self.rank * self.n:(self.rank + 1) * self.n, :]

    def forward(self, q0: torch.Tensor, n_steps: int) -> torch.Tensor:
        """Advance this slab's interior state q0 [4, n, nx] by n_steps steps
        (every rank the same n_steps), recording the run; returns the final
        interior rows. The x ghosts are filled periodically here and the y
        ghosts by the exchange."""
        ng = self.ng
        self.qpad = pad_periodic(q0.detach().to(torch.float64), ng)
        clk = capi.McClock()
        clk.time, clk.max_time = 0.0, 1e300
        clk.prev_output_time, clk.output_delta = 0.0, 1e300
        self._check(self.lib.mc_adjoint_forward(self.h, ctypes.c_void_p(self.qpad.data_ptr()), ctypes.byref(clk),
                                                int(n_steps), self._stream()), "mc_adjoint_forward")
        return self.qpad[:, 0, ng:-ng, ng:-ng].clone()

    def backward(self, lam: torch.Tensor):
        """lam: dJ/d(final interior rows of this slab) [4, n, nx]. Returns
        (dJ/d(initial interior rows) [4, n, nx], dJ/dgamma summed over the
        ranks)."""
        ng = self.ng
        lpad = torch.zeros_like(self.qpad)
        lpad[:, 0, ng:-ng, ng:-ng] = lam.to(torch.float64)
        g = ctypes.c_double()
        self._check(self.lib.mc_adjoint_backward(self.h, ctypes.c_void_p(lpad.data_ptr()), ctypes.byref(g),
                                                 self._stream()), "mc_adjoint_backward")
        return lpad[:, 0, ng:-ng, ng:-ng].clone(), g.value


def kh_initial_state(vy: torch.Tensor, gamma: torch.Tensor, problem: Problem) -> torch.Tensor:
    """Interior conserved KH state [4, n, n] from the vy field [n, n] (the
    band densities / velocities / pressure of ``problems.kelvin_helmholtz_2d``),
    with the reference's prim_to_cons order (source/Eos.hpp:81-99)."""
    n, ng, dx = problem.nx, problem.ng, problem.dx
    x = (torch.arange(n, dtype=torch.float64, device=vy.device) + 0.5) * dx
    Y = x.view(n, 1).expand(n, n)
    band = (Y - 0.5).abs() < 0.25
    rho = torch.where(band, torch.tensor(2.0, dtype=torch.float64, device=vy.device),
                      torch.tensor(1.0, dtype=torch.float64, device=vy.device))
    vx = torch.where(band, torch.tensor(0.5, dtype=torch.float64, device=vy.device),
                     torch.tensor(-0.5, dtype=torch.float64, device=vy.device))
    p = torch.full_like(rho, 2.5)
    mx = rho * vx
    my = rho * vy
    v2 = vx * vx + vy * vy
    e = p / (gamma - 1.0) + (0.5 * rho) * v2
    return torch.stack([rho, mx, my, e])


def kh_vy(problem: Problem) -> np.ndarray:
    """The interior vy field of a KH Problem's initial state."""
    ng = problem.ng
    q = problem.Q[:, 0, ng:-ng, ng:-ng]
    return q[2] / q[0]


def tangent_linear(problem: Problem, q0: torch.Tensor, gamma: float, dq0: torch.Tensor, dgamma, n_steps: int):
    """Forward-mode derivative of ``n_steps`` steps (``mc_tangent_linear``):
    ``q0`` the interior state [4, ny, nx], ``dq0`` k tangent states
    [k, 4, ny, nx], ``dgamma`` k tangents of gamma. Returns the final
    interior state (bit-identical to ``EulerSteps``' forward run) and the k
    final tangents [k, 4, ny, nx]."""
    lib = capi.load()
    ng = problem.ng
    k = int(dq0.shape[0])
    qpad = pad_periodic(q0.detach().to(torch.float64), ng)
    dpad = torch.stack([pad_periodic(dq0[i].detach().to(torch.float64), ng) for i in range(k)]).contiguous()
    grid = grid_of(problem)
    scheme = _scheme(problem, gamma)
    clk = capi.McClock()
    clk.time, clk.max_time = 0.0, 1e300
    clk.prev_output_time, clk.output_delta = 0.0, 1e300
    dg = (ctypes.c_double * k)(*[float(x) for x in dgamma])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(lib.mc_tangent_linear(ctypes.byref(grid), ctypes.byref(scheme), ctypes.c_void_p(qpad.data_ptr()),
                                     ctypes.c_void_p(dpad.data_ptr()), dg, k, ctypes.byref(clk), int(n_steps),
                                     stream), "mc_tangent_linear")
    return qpad[:, 0, ng:-ng, ng:-ng].clone(), dpad[:, :, 0, ng:-ng, ng:-ng].clone()


def kh_directional_derivatives(problem: Problem, vy: torch.Tensor, gamma: float, dvy: torch.Tensor, dgamma,
                               rho_target: torch.Tensor, n_steps: int):
    """Directional derivatives of J = 1/2 |rho_final - rho_target|^2 along
    the directions (dvy[k], dgamma[k]) of (initial vy field, gamma) by the
    tangent-linear model: the initial tangents are the forward-mode
    derivatives of kh_initial_state; returns (J, [dJ_k])."""
    with torch.no_grad():
        g = torch.tensor(gamma, dtype=torch.float64, device=vy.device)
        q0 = kh_initial_state(vy, g, problem)
        dq0 = []
        for k in range(dvy.shape[0]):
            tg = torch.tensor(float(dgamma[k]), dtype=torch.float64, device=vy.device)
            dq0.append(torch.func.jvp(lambda v, gg: kh_initial_state(v, gg, problem), (vy, g), (dvy[k], tg))[1])
        qn, dqn = tangent_linear(problem, q0, gamma, torch.stack(dq0), dgamma, n_steps)
        r = qn[0] - rho_target
        J = 0.5 * float((r * r).sum())
        dJ = [float((r * dqn[k, 0]).sum()) for k in range(dqn.shape[0])]
    return J, dJ
