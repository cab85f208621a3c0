"""Oracle test infrastructure, not product code.

ctypes access to the two CPU implementations of Mosscap's hydro step that
serve as the correctness checker:

* ``kind="reference"``: ``oracle/_ref/libmosscap_ref.so`` -- the reference's
  own ``source/Hydro.cpp`` and ``source/TimeStepping.cpp`` compiled unmodified
  against the host Kokkos/YAKL shim (``oracle/ref_shim``), driven by
  ``oracle/ref_harness.cpp``;
* ``kind="port"``: ``oracle/liboracle_port.so`` -- the plain-C restatement in
  ``oracle/mosscap_oracle.c``.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference's source tree (its ``source/`` directory), read only when the
# reference build is made; MOSSCAP_REFERENCE_SOURCE overrides the default.
REF_SOURCE = os.environ.get("MOSSCAP_REFERENCE_SOURCE", "/root/reference/source")
LIB_PATHS = {
    "reference": os.path.join(HERE, "_ref", "libmosscap_ref.so"),
    "port": os.path.join(HERE, "liboracle_port.so"),
}
# The adapter check program (oracle/adapter_check.cpp), built with the reference.
ADAPTER_CHECK = os.path.join(HERE, "_ref", "adapter_check")

# Reference enum ordinals (source/Reconstruct.hpp:10-27, source/Riemann.hpp:10-14,
# source/TimeStepping.hpp:10-14, source/State.hpp:62-70).
RECON = {"fog": 0, "muscl": 1, "ppm": 2, "weno5z": 3}
LIMITER = {"vanleer": 0, "monotonizedcentral": 1, "minmod": 2}
RIEMANN = {"rusanov": 0, "hll": 1, "hllc": 2}
STEPPER = {"rk2": 0, "ssprk3": 1, "ssprk4": 2}
BOUNDARY = {"wall": 0, "periodic": 1, "symmetric": 2, "symmetricoutflowdiode": 3,
            "zerograd": 4, "constant": 5, "userfn": 6}


class _Config(ctypes.Structure):
    _fields_ = [
        ("num_dim", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("ng", ctypes.c_int32),
        ("num_tracers", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("loc", ctypes.c_double * 3),
        ("bc", ctypes.c_int32 * 6),
        ("bc_const", (ctypes.c_double * 5) * 6),
        ("reconstruction", ctypes.c_int32), ("slope_limiter", ctypes.c_int32),
        ("riemann_solver", ctypes.c_int32), ("time_stepper", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("max_cfl", ctypes.c_double),
        ("max_time", ctypes.c_double),
        ("output_delta", ctypes.c_double),
    ]


class EosTable(ctypes.Structure):
    """moracle_eos_table: the tabulated LTE hydrogen EOS grid and tables."""
    _fields_ = [
        ("log_eint_rho_start", ctypes.c_double), ("log_eint_rho_step", ctypes.c_double),
        ("n_eint_rho", ctypes.c_int32),
        ("log_rho_start", ctypes.c_double), ("log_rho_step", ctypes.c_double),
        ("n_rho", ctypes.c_int32),
        ("y_table", ctypes.POINTER(ctypes.c_double)),
        ("log_T_table", ctypes.POINTER(ctypes.c_double)),
    ]


EOS_TYPE = {"ideal": 0, "analyticlteh": 1, "tabulatedlteh": 2}


def build(kind: str = "all") -> None:
    """Build the oracle libraries with ``oracle/Makefile`` (``make port|ref|adapter``;
    ``adapter`` links the product library, which must be built first)."""
    targets = ["port", "ref", "adapter"] if kind == "all" else [kind]
    subprocess.run(["make", "-s", "-C", HERE, f"REF_SRC={REF_SOURCE}"] + targets, check=True)


def have_reference_sources() -> bool:
    """Whether the reference's source tree is present (it is not on every
    machine that runs the tests; the built libraries travel instead)."""
    return os.path.isdir(REF_SOURCE)


_LIBS: dict = {}


def load(kind: str) -> ctypes.CDLL:
    if kind in _LIBS:
        return _LIBS[kind]
    path = LIB_PATHS[kind]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
    lib = ctypes.CDLL(path)
    vp, d, i64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int64
    dptr = ctypes.POINTER(ctypes.c_double)
    lib.moracle_create.argtypes = [ctypes.POINTER(_Config)]
    lib.moracle_create.restype = vp
    lib.moracle_destroy.argtypes = [vp]
    lib.moracle_state_size.argtypes = [vp]
    lib.moracle_state_size.restype = i64
    for name in ("moracle_set_Q", "moracle_get_Q", "moracle_get_W"):
        getattr(lib, name).argtypes = [vp, dptr]
    lib.moracle_fill_bcs.argtypes = [vp]
    lib.moracle_compute_dt.argtypes = [vp]
    lib.moracle_compute_dt.restype = d
    lib.moracle_cfl_min.argtypes = [vp]
    lib.moracle_cfl_min.restype = d
    lib.moracle_time_step.argtypes = [vp, d]
    lib.moracle_run.argtypes = [vp, i64, dptr]
    lib.moracle_run.restype = i64
    lib.moracle_get_time.argtypes = [vp]
    lib.moracle_get_time.restype = d
    lib.moracle_set_clock.argtypes = [vp, d, d]
    lib.moracle_set_num_threads.argtypes = [ctypes.c_int]
    lib.moracle_set_gravity.argtypes = [vp, ctypes.c_int, d, d, d]
    lib.moracle_set_eos.argtypes = [vp, ctypes.c_int, d, ctypes.c_int, ctypes.POINTER(EosTable)]
    lib.moracle_set_eos.restype = ctypes.c_int
    lib.moracle_update_eos.argtypes = [vp]
    lib.moracle_get_eos_fields.argtypes = [vp, dptr, dptr]
    lib.moracle_abort_count.restype = ctypes.c_longlong
    _LIBS[kind] = lib
    return lib


@dataclass
class OracleConfig:
    """Grid + scheme description, mirroring the reference's Simulation setup."""
    num_dim: int
    nx: int
    ny: int = 1
    nz: int = 1
    ng: int = 3
    num_tracers: int = 0
    dx: float = 1.0
    loc: Sequence[float] = (0.0, 0.0, 0.0)
    bc: Sequence[str] = ("zerograd",) * 6
    bc_const: Optional[np.ndarray] = None
    reconstruction: str = "muscl"
    slope_limiter: str = "monotonizedcentral"
    riemann_solver: str = "hll"
    time_stepper: str = "ssprk3"
    gamma: float = 1.4
    max_cfl: float = 0.8
    max_time: float = 1.0
    output_delta: float = 0.1

    def to_c(self) -> _Config:
        c = _Config()
        c.num_dim = self.num_dim
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.ng = self.ng
        c.num_tracers = self.num_tracers
        c.dx = self.dx
        for a in range(3):
            c.loc[a] = self.loc[a]
        for f in range(6):
            c.bc[f] = BOUNDARY[self.bc[f]]
        if self.bc_const is not None:
            bcc = np.asarray(self.bc_const, dtype=np.float64).reshape(6, 5)
            for f in range(6):
                for v in range(5):
                    c.bc_const[f][v] = bcc[f, v]
        c.reconstruction = RECON[self.reconstruction]
        c.slope_limiter = LIMITER[self.slope_limiter]
        c.riemann_solver = RIEMANN[self.riemann_solver]
        c.time_stepper = STEPPER[self.time_stepper]
        c.gamma = self.gamma
        c.max_cfl = self.max_cfl
        c.max_time = self.max_time
        c.output_delta = self.output_delta
        return c

    @property
    def n_vars(self) -> int:
        return 2 + self.num_dim + self.num_tracers

    @property
    def shape(self):
        """Q shape ``[var][zc][yc][xc]`` (the reference layout, i fastest)."""
        xc = self.nx + 2 * self.ng
        yc = self.ny + 2 * self.ng if self.num_dim > 1 else 1
        zc = self.nz + 2 * self.ng if self.num_dim > 2 else 1
        return (self.n_vars, zc, yc, xc)


class OracleSim:
    """One Simulation held by an oracle library."""

    def __init__(self, cfg: OracleConfig, kind: str = "reference", threads: int = 0):
        self.lib = load(kind)
        self.kind = kind
        self.cfg = cfg
        if threads:
            self.lib.moracle_set_num_threads(int(threads))
        self._c = cfg.to_c()
        self.h = self.lib.moracle_create(ctypes.byref(self._c))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        assert self.lib.moracle_state_size(self.h) == int(np.prod(cfg.shape))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.moracle_destroy(h)
            self.h = None

    @staticmethod
    def _ptr(a: np.ndarray):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def set_Q(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == self.cfg.shape
        self.lib.moracle_set_Q(self.h, self._ptr(q))

    def get_Q(self) -> np.ndarray:
        q = np.empty(self.cfg.shape, dtype=np.float64)
        self.lib.moracle_get_Q(self.h, self._ptr(q))
        return q

    def get_W(self) -> np.ndarray:
        w = np.empty(self.cfg.shape, dtype=np.float64)
        self.lib.moracle_get_W(self.h, self._ptr(w))
        return w

    def fill_bcs(self) -> None:
        self.lib.moracle_fill_bcs(self.h)

    def compute_dt(self) -> float:
        return self.lib.moracle_compute_dt(self.h)

    def cfl_min(self) -> float:
        return self.lib.moracle_cfl_min(self.h)

    def time_step(self, dt: float) -> None:
        self.lib.moracle_time_step(self.h, dt)

    def run(self, max_steps: int) -> np.ndarray:
        log = np.zeros(max(int(max_steps), 1), dtype=np.float64)
        n = self.lib.moracle_run(self.h, int(max_steps), self._ptr(log))
        return log[:n].copy()

    @property
    def time(self) -> float:
        return self.lib.moracle_get_time(self.h)

    def set_clock(self, time: float, prev_output_time: float) -> None:
        self.lib.moracle_set_clock(self.h, time, prev_output_time)

    def set_eos(self, kind: str, avg_mass: float = 1.0, include_ionisation_energy: bool = False,
                table=None) -> None:
        """Select the EOS: "ideal", "analyticlteh" or "tabulatedlteh"; table =
        (log_eint_rho_start, log_eint_rho_step, log_rho_start, log_rho_step,
        y_table [n_rho, n_eint_rho], log_T_table [n_rho, n_eint_rho])."""
        tab = None
        if table is not None:
            xs, xd, ys, yd, yt, lt = table
            self._eos_y = np.ascontiguousarray(yt, dtype=np.float64)
            self._eos_t = np.ascontiguousarray(lt, dtype=np.float64)
            tab = EosTable(xs, xd, self._eos_y.shape[1], ys, yd, self._eos_y.shape[0], self._ptr(self._eos_y),
                           self._ptr(self._eos_t))
        r = self.lib.moracle_set_eos(self.h, EOS_TYPE[kind], float(avg_mass), int(include_ionisation_energy),
                                     ctypes.byref(tab) if tab is not None else None)
        if r != 0:
            raise ValueError("oracle rejected the EOS")

    def update_eos(self) -> None:
        self.lib.moracle_update_eos(self.h)

    def eos_fields(self):
        """(y, T), each [zc, yc, xc]."""
        shape = self.cfg.shape[1:]
        y = np.empty(shape, dtype=np.float64)
        T = np.empty(shape, dtype=np.float64)
        self.lib.moracle_get_eos_fields(self.h, self._ptr(y), self._ptr(T))
        return y, T

    def abort_count(self) -> int:
        return int(self.lib.moracle_abort_count())

    def set_gravity(self, g) -> None:
        """Register the gravity source term with acceleration g = (gx, gy, gz);
        None removes it."""
        if g is None:
            self.lib.moracle_set_gravity(self.h, 0, 0.0, 0.0, 0.0)
        else:
            self.lib.moracle_set_gravity(self.h, 1, float(g[0]), float(g[1]), float(g[2]))
