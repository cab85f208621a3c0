"""Host-side mirror of the hydro part of Mosscap's ``Simulation``.

:class:`HydroSim` holds the conserved state ``Q`` on the GPU (a float64 torch
tensor in the reference layout ``[var][zc][yc][xc]``) together with the clock
of ``Simulation``/``OutputConfig``, and exposes the reference's hooks with
their names and meaning:

=====================  ==========================================  =========================
reference              here                                        C ABI
=====================  ==========================================  =========================
``fill_bcs(sim)``      :meth:`HydroSim.fill_bcs`                   ``mc_fill_bcs``
``sim.compute_dt``     :meth:`HydroSim.compute_dt` (with clamp)    ``mc_compute_dt``
``sim.time_step``      :meth:`HydroSim.time_step` (``time += dt``) ``mc_time_step``
main loop              :meth:`HydroSim.run` / :meth:`advance`      ``mc_advance``
=====================  ==========================================  =========================

(``source/Boundaries.hpp:132-149``, ``source/Hydro.cpp:345``,
``source/TimeStepping.cpp:39-308``, ``source/main.cpp:54-72``.)

torch provides device memory and streams only; every computation is a kernel
of ``libmosscap_b200.so``.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import capi
from .problems import Problem


class HydroSim:
    def __init__(self, problem: Problem, precision: str = "fp64", device: Optional[torch.device] = None,
                 Q: Optional[np.ndarray] = None):
        self.lib = capi.load()
        self.problem = problem
        self.device = torch.device(device or "cuda")
        p = problem
        shape = p.shape
        g = capi.McGrid()
        g.num_dim = p.num_dim
        g.zc, g.yc, g.xc = shape[1], shape[2], shape[3]
        g.ng = p.ng
        g.num_tracers = p.num_tracers
        g.dx = p.dx
        for a in range(3):
            g.loc[a] = p.loc[a]
        for f in range(6):
            g.bc[f] = capi.BOUNDARY[p.bc[f]]
        if p.bc_const is not None:
            bcc = np.asarray(p.bc_const, dtype=np.float64).reshape(6, 5)
            for f in range(6):
                for v in range(5):
                    g.bc_const[f][v] = bcc[f, v]
        s = capi.McScheme()
        s.reconstruction = capi.RECON[p.reconstruction]
        s.slope_limiter = capi.LIMITER[p.slope_limiter]
        s.riemann_solver = capi.RIEMANN[p.riemann_solver]
        s.time_stepper = capi.STEPPER[p.time_stepper]
        s.precision = capi.PRECISION[precision]
        s.gamma = p.gamma
        s.max_cfl = p.max_cfl
        self._grid, self._scheme = g, s
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            capi.check(self.lib.mc_create(ctypes.byref(g), ctypes.byref(s), ctypes.byref(h)), "mc_create")
        self.ctx = h
        if p.gravity is not None:
            gx, gy, gz = (float(x) for x in p.gravity)
            capi.check(self.lib.mc_set_gravity(h, 1, gx, gy, gz), "mc_set_gravity")
        if p.eos != "ideal":
            tab = None
            if p.eos_table is not None:
                xs, xd, ys, yd, yt, lt = p.eos_table
                self._eos_y = np.ascontiguousarray(yt, dtype=np.float64)
                self._eos_t = np.ascontiguousarray(lt, dtype=np.float64)
                dp = ctypes.POINTER(ctypes.c_double)
                tab = capi.McEosTable(xs, xd, self._eos_y.shape[1], ys, yd, self._eos_y.shape[0],
                                      self._eos_y.ctypes.data_as(dp), self._eos_t.ctypes.data_as(dp))
            with torch.cuda.device(self.device):
                capi.check(self.lib.mc_set_eos(h, capi.EOS[p.eos], float(p.eos_avg_mass), int(p.eos_ionisation),
                                               ctypes.byref(tab) if tab is not None else None), "mc_set_eos")
        q = Q if Q is not None else p.Q
        if q is None:
            raise ValueError("no initial state")
        self.Q = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float64)).to(self.device)
        assert tuple(self.Q.shape) == tuple(shape)
        # Simulation::time and the OutputConfig clock; setup_sim writes the
        # initial conditions at time 0 (source/SetupModules.hpp:258-259)
        self.time = 0.0
        self.max_time = p.max_time
        self.output_delta = p.output_delta
        self.prev_output_time = 0.0
        self.current_step = 0

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.lib.mc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- plumbing ---------------------------------------------------------
    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _qptr(self, q: Optional[torch.Tensor] = None) -> ctypes.c_void_p:
        q = self.Q if q is None else q
        assert q.is_cuda and q.dtype == torch.float64 and q.is_contiguous()
        return ctypes.c_void_p(q.data_ptr())

    def _clock(self) -> capi.McClock:
        c = capi.McClock()
        c.time, c.max_time = self.time, self.max_time
        c.prev_output_time, c.output_delta = self.prev_output_time, self.output_delta
        return c

    # ---- the reference's hooks ----------------------------------------------
    def fill_bcs(self) -> None:
        capi.check(self.lib.mc_fill_bcs(self.ctx, self._qptr(), self._stream()), "mc_fill_bcs")

    def compute_dt(self, clamp: bool = True) -> float:
        dt = ctypes.c_double()
        clk = self._clock()
        capi.check(self.lib.mc_compute_dt(self.ctx, self._qptr(), ctypes.byref(clk) if clamp else None,
                                          ctypes.byref(dt), self._stream()), "mc_compute_dt")
        return dt.value

    def time_step(self, dt: float) -> None:
        capi.check(self.lib.mc_time_step(self.ctx, self._qptr(), float(dt), self._stream()), "mc_time_step")
        self.time += dt
        self.current_step += 1

    def step_host(self, q_host: torch.Tensor, clamp: bool = True) -> float:
        """compute_dt + time_step on a host-resident state (mc_step_host):
        q_host (float64 CPU tensor of Q's shape, pinned for the copies to
        overlap the step) goes to the device copy Q, one step is taken there
        and the result returns to q_host. Advances the clock like time_step;
        returns dt."""
        assert q_host.device.type == "cpu" and q_host.dtype == torch.float64 and q_host.is_contiguous()
        assert tuple(q_host.shape) == tuple(self.Q.shape)
        dt = ctypes.c_double()
        clk = self._clock()
        capi.check(self.lib.mc_step_host(self.ctx, ctypes.c_void_p(q_host.data_ptr()), self._qptr(),
                                         ctypes.byref(clk) if clamp else None, ctypes.byref(dt), self._stream()),
                   "mc_step_host")
        self.time += dt.value
        self.current_step += 1
        return dt.value

    def last_cfl_min(self) -> float:
        v = ctypes.c_double()
        capi.check(self.lib.mc_last_cfl_min(self.ctx, ctypes.byref(v), self._stream()), "mc_last_cfl_min")
        return v.value

    def update_eos(self) -> None:
        """One EOS update of Q (Simulation::update_eos, as setup_sim calls it
        before the first step, source/SetupModules.hpp:253-255)."""
        capi.check(self.lib.mc_update_eos(self.ctx, self._qptr(), self._stream()), "mc_update_eos")

    def eos_fields(self):
        """The ionisation fraction and temperature fields of the last EOS
        update (y_space, T_space), each [zc, yc, xc]."""
        shape = tuple(self.Q.shape[1:])
        y = torch.empty(shape, dtype=torch.float64, device=self.device)
        T = torch.empty(shape, dtype=torch.float64, device=self.device)
        capi.check(self.lib.mc_get_eos_fields(self.ctx, ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(T.data_ptr()),
                                              self._stream()), "mc_get_eos_fields")
        torch.cuda.synchronize(self.device)
        return y.cpu().numpy(), T.cpu().numpy()

    def get_W(self) -> np.ndarray:
        """The primitive state the reference's State.W holds after its last
        time_step (the last stage's input through global_cons_to_prim,
        source/Hydro.cpp:8-53), ghosts included; before the first step, the
        primitives of Q (mc_get_prim)."""
        W = torch.empty_like(self.Q)
        capi.check(self.lib.mc_get_prim(self.ctx, self._qptr(), ctypes.c_void_p(W.data_ptr()), self._stream()),
                   "mc_get_prim")
        torch.cuda.synchronize(self.device)
        return W.cpu().numpy()

    def status(self) -> int:
        f = ctypes.c_uint32()
        capi.check(self.lib.mc_get_status(self.ctx, ctypes.byref(f), self._stream()), "mc_get_status")
        return f.value

    def profile_stages(self, enable: bool) -> None:
        capi.check(self.lib.mc_profile_stages(self.ctx, int(bool(enable))), "mc_profile_stages")

    def stage_time(self, kind: int = 0):
        """(summed ms, launches) of the stage kernels recorded since
        profile_stages(True)."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        capi.check(self.lib.mc_stage_time(self.ctx, int(kind), ctypes.byref(ms), ctypes.byref(n)), "mc_stage_time")
        return ms.value, n.value

    def launch_count(self) -> int:
        return int(self.lib.mc_launch_count(self.ctx))

    # ---- main loop --------------------------------------------------------
    def advance(self, max_steps: int, log_dt: bool = True) -> np.ndarray:
        """Device-driven loop (mc_advance); stops after max_steps, at max_time
        or after a step that makes an output due. Returns the dt of each step."""
        clk = self._clock()
        done = ctypes.c_int64()
        log = np.zeros(max(int(max_steps), 1), dtype=np.float64)
        capi.check(self.lib.mc_advance(self.ctx, self._qptr(), ctypes.byref(clk), int(max_steps),
                                       ctypes.byref(done),
                                       log.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if log_dt else None,
                                       self._stream()), "mc_advance")
        self.time = clk.time
        self.prev_output_time = clk.prev_output_time
        self.current_step += done.value
        return log[:done.value].copy()

    def run(self, max_steps: int = 1 << 62, device_loop: bool = True, output=None) -> np.ndarray:
        """The main loop of source/main.cpp:54-72. Without `output` (an
        :class:`~mosscap_b200.output.OutputConfig`) outputs only move the
        clock; with it, the files of source/Output.cpp are written: first the
        initial output if none has been written yet (setup_sim,
        source/SetupModules.hpp:259), then one after every step that makes
        an output due, and a last one when the loop ends."""
        from .output import write_output
        if output is not None and output.prev_output_time < 0.0:
            write_output(self, output)
        dts = []
        n = 0
        while self.time < self.max_time and n < max_steps:
            if device_loop:
                # the dt log of one call is host memory: bounded chunks
                d = self.advance(min(max_steps - n, 1 << 16))
                dts.extend(d.tolist())
                n += len(d)
                if len(d) == 0:
                    break
            else:
                dt = self.compute_dt()
                self.time_step(dt)
                dts.append(dt)
                n += 1
                if self.time >= self.prev_output_time + self.output_delta:
                    self.prev_output_time = self.time
            if output is not None and self.time >= output.prev_output_time + self.output_delta:
                write_output(self, output)
        if output is not None:
            write_output(self, output)
        return np.asarray(dts)

    def get_Q(self) -> np.ndarray:
        return self.Q.detach().cpu().numpy()


def grid_of(p: Problem) -> capi.McGrid:
    """The mc_grid of a Problem."""
    g = capi.McGrid()
    shape = p.shape
    g.num_dim = p.num_dim
    g.zc, g.yc, g.xc = shape[1], shape[2], shape[3]
    g.ng = p.ng
    g.num_tracers = p.num_tracers
    g.dx = p.dx
    for a in range(3):
        g.loc[a] = p.loc[a]
    for f in range(6):
        g.bc[f] = capi.BOUNDARY[p.bc[f]]
    return g


class BatchSim:
    """Many independent 1D / 2D problems advanced together (mc_batch_*).

    The problems' states live in one float64 pool on the GPU, each problem's
    ``[var][zc][yc][xc]`` block at its own offset. Every problem runs its own
    main loop with its own dt; ``advance(k)`` replays the captured step graph
    k times."""

    def __init__(self, problems: Sequence[Problem], precision: str = "fp64",
                 device: Optional[torch.device] = None):
        self.lib = capi.load()
        self.device = torch.device(device or "cuda")
        self.problems = list(problems)
        p0 = self.problems[0]
        offs, total = [], 0
        for p in self.problems:
            offs.append(total)
            total += int(np.prod(p.shape))
            total = (total + 31) // 32 * 32  # 256-byte aligned blocks
        self.offsets = offs
        pool = np.zeros(total, dtype=np.float64)
        for p, o in zip(self.problems, offs):
            pool[o:o + int(np.prod(p.shape))] = np.ascontiguousarray(p.Q, dtype=np.float64).ravel()
        self.pool = torch.from_numpy(pool).to(self.device)
        arr = (capi.McBatchProblem * len(self.problems))()
        for k, (p, o) in enumerate(zip(self.problems, offs)):
            arr[k].grid = grid_of(p)
            arr[k].offset = o
            arr[k].max_cfl = p.max_cfl
            arr[k].clock.time = 0.0
            arr[k].clock.max_time = p.max_time
            arr[k].clock.prev_output_time = 0.0
            arr[k].clock.output_delta = p.output_delta
        s = capi.McScheme()
        s.reconstruction = capi.RECON[p0.reconstruction]
        s.slope_limiter = capi.LIMITER[p0.slope_limiter]
        s.riemann_solver = capi.RIEMANN[p0.riemann_solver]
        s.time_stepper = capi.STEPPER[p0.time_stepper]
        s.precision = capi.PRECISION[precision]
        s.gamma = p0.gamma
        s.max_cfl = p0.max_cfl
        self._problems_c, self._scheme = arr, s
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            capi.check(self.lib.mc_batch_create(arr, len(self.problems), ctypes.byref(s), total, ctypes.byref(h)),
                       "mc_batch_create")
        self.ctx = h

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.lib.mc_batch_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _pool(self):
        return ctypes.c_void_p(self.pool.data_ptr())

    def fill_bcs(self) -> None:
        capi.check(self.lib.mc_batch_fill_bcs(self.ctx, self._pool(), self._stream()), "mc_batch_fill_bcs")

    def tune(self):
        capi.check(self.lib.mc_batch_tune(self.ctx, self._pool(), self._stream()), "mc_batch_tune")
        return self.schedule()

    def schedule(self):
        g, d, s = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        capi.check(self.lib.mc_batch_schedule(self.ctx, ctypes.byref(g), ctypes.byref(d), ctypes.byref(s)),
                   "mc_batch_schedule")
        n = ctypes.c_int32()
        capi.check(self.lib.mc_batch_stage_launches(self.ctx, ctypes.byref(n)), "mc_batch_stage_launches")
        return {"grid": g.value, "dynamic": bool(d.value), "segments_per_task": s.value,
                "launches_per_stage": n.value}

    def set_stage_launches(self, n: int) -> None:
        """1: one launch per stage over all work items; 2: the 2D tiles and
        the 1D tasks in separate launches (until the next tune())."""
        capi.check(self.lib.mc_batch_set_stage_launches(self.ctx, int(n)), "mc_batch_set_stage_launches")

    def advance(self, steps: int) -> None:
        capi.check(self.lib.mc_batch_advance(self.ctx, self._pool(), int(steps), self._stream()), "mc_batch_advance")

    def clocks(self):
        n = len(self.problems)
        clk = (capi.McClock * n)()
        steps = (ctypes.c_int64 * n)()
        status = (ctypes.c_uint32 * n)()
        capi.check(self.lib.mc_batch_clocks(self.ctx, clk, steps, status, self._stream()), "mc_batch_clocks")
        return (np.array([c.time for c in clk]), np.array(list(steps)), np.array(list(status)))

    def get_Q(self, k: int) -> np.ndarray:
        p = self.problems[k]
        n = int(np.prod(p.shape))
        return self.pool[self.offsets[k]:self.offsets[k] + n].view(p.shape).cpu().numpy()
