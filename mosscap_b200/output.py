"""Simulation output in the reference's NetCDF layout (source/Output.cpp).

:func:`write_output` mirrors ``write_output`` (source/Output.cpp:194-277)
with the configuration of ``setup_output`` (source/SetupModules.hpp:179-194):

* global attributes ``hydro_program``, ``hydro_git_hash``, ``problem``,
  ``num_ghost``, ``single_file``, ``write_conserved``, ``write_primitive``,
  ``write_fluxes``, ``write_source_term`` and the variable indices
  (``irho``, ``imx`` ... ``iene``; ``ivx`` ... ``ipre``), in that order
  (source/Output.cpp:18-157);
* dimensions ``x``, ``y``, ``z`` (cells including ghosts) and the cell-centre
  coordinates ``x`` (``y``, ``z`` in 2D / 3D) of State::get_pos
  (source/State.hpp:123-134), then ``time`` (source/Output.cpp:159-192);
* ``Q`` and, if asked for, ``W`` over ``(var, z, y, x)``, and for a
  non-ideal EOS ``ion_frac`` and ``T`` over ``(z, y, x)``;
* one file per output (``<name>_NNNNN.nc``, a ``time`` dimension of one) or,
  the reference's default, one file (``<name>.nc``) with ``time`` unlimited
  and one record per output.

``W`` is what the reference's State.W holds at output time: the primitives
of the last stage's input (:meth:`HydroSim.get_W`). Face fluxes and the
source-term array are never stored by the fused stage kernels, so
``fluxes`` / ``source`` output is refused with an error.

The files are NetCDF classic format (CDF-1, or CDF-2 / CDF-5 when offsets
or a variable pass the 32-bit limits: a 512^3 five-variable Q is 5.6 GB);
the reference's files come from the netCDF library's default format, which
is also CDF-1 for nc_create with NC_CLOBBER.
"""
from __future__ import annotations

import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import netcdf as nc


@dataclass
class OutputVariables:
    """OutputOptions (source/Output.hpp:9-14)."""
    conserved: bool = True
    primitive: bool = False
    fluxes: bool = False
    source: bool = False


@dataclass
class OutputConfig:
    """OutputConfig (source/Output.hpp:16-24), defaults of setup_output
    (source/SetupModules.hpp:179-190)."""
    filename: str
    problem_name: str
    single_file: bool = True
    output_count: int = 0
    delta: float = 0.1
    prev_output_time: float = -1.0
    variables: OutputVariables = field(default_factory=OutputVariables)
    directory: str = "."

    @classmethod
    def for_problem(cls, problem, name: Optional[str] = None, **kw) -> "OutputConfig":
        """output.name defaults to output_<problem name>."""
        return cls(filename=name or f"output_{problem.name}", problem_name=problem.name,
                   delta=problem.output_delta, **kw)


def _git_hash() -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    try:
        r = subprocess.run(["git", "-C", here, "rev-parse", "HEAD"], capture_output=True, text=True, timeout=10)
        if r.returncode == 0:
            return r.stdout.strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return "unknown"


def cell_centres(n: int, ng: int, dx: float, loc: float) -> np.ndarray:
    """get_pos along one axis: i * dx + (-(ng - 0.5) * dx) + loc."""
    ghost_offset = -(ng - 0.5) * dx
    return (np.arange(n, dtype=np.float64) * dx + ghost_offset) + loc


def _header(w: nc.NcWriter, cfg: OutputConfig, num_dim: int, ng: int) -> None:
    v = cfg.variables
    w.put_att("hydro_program", "mosscap")
    w.put_att("hydro_git_hash", _git_hash())
    w.put_att("problem", cfg.problem_name)
    w.put_att("num_ghost", int(ng))
    w.put_att("single_file", int(cfg.single_file))
    w.put_att("write_conserved", int(v.conserved))
    w.put_att("write_primitive", int(v.primitive))
    w.put_att("write_fluxes", int(v.fluxes))
    w.put_att("write_source_term", int(v.source))
    axes = "xyz"[:num_dim]
    if v.conserved:
        w.put_att("irho", 0)
        for a, name in enumerate(axes):
            w.put_att(f"im{name}", 1 + a)
        w.put_att("iene", 1 + num_dim)
    if v.primitive:
        w.put_att("irho", 0)
        for a, name in enumerate(axes):
            w.put_att(f"iv{name}", 1 + a)
        w.put_att("ipre", 1 + num_dim)


def write_output(sim, cfg: OutputConfig) -> bool:
    """One output of `sim` (a :class:`~mosscap_b200.hydro.HydroSim`, or any
    object with ``problem``, ``time``, ``get_Q()``, ``get_W()`` and, for a
    non-ideal EOS, ``eos_fields()``)."""
    v = cfg.variables
    if v.fluxes or v.source:
        raise NotImplementedError("fluxes / source output: the fused stage kernels do not store face fluxes "
                                  "or the source-term array")
    p = sim.problem
    nvar, zc, yc, xc = p.shape
    non_ideal = getattr(p, "eos", "ideal") != "ideal"
    if cfg.single_file:
        path = os.path.join(cfg.directory, f"{cfg.filename}.nc")
    else:
        path = os.path.join(cfg.directory, f"{cfg.filename}_{cfg.output_count:05d}.nc")
    data = {}
    if v.conserved:
        data["Q"] = sim.get_Q()
    if v.primitive:
        data["W"] = sim.get_W()
    if non_ideal:
        y, T = sim.eos_fields()
        data["ion_frac"], data["T"] = y, T
    fields = [k for k in ("Q", "W", "ion_frac", "T") if k in data]

    if cfg.prev_output_time < 0.0 or not cfg.single_file:
        w = nc.NcWriter(path)
        _header(w, cfg, p.num_dim, p.ng)
        w.create_dim("x", xc)
        w.create_dim("y", yc)
        w.create_dim("z", zc)
        w.def_var("x", ["x"])
        if p.num_dim > 1:
            w.def_var("y", ["y"])
        if p.num_dim > 2:
            w.def_var("z", ["z"])
        w.create_dim("time", None if cfg.single_file else 1)
        lead = ["time"] if cfg.single_file else []
        w.def_var("time", ["time"])
        if "Q" in data or "W" in data:
            w.create_dim("var", nvar)
        for k in fields:
            w.def_var(k, lead + (["var", "z", "y", "x"] if k in ("Q", "W") else ["z", "y", "x"]))
        w.end_def()
        w.write("x", cell_centres(xc, p.ng, p.dx, p.loc[0]))
        if p.num_dim > 1:
            w.write("y", cell_centres(yc, p.ng, p.dx, p.loc[1]))
        if p.num_dim > 2:
            w.write("z", cell_centres(zc, p.ng, p.dx, p.loc[2]))
    else:
        w = nc.NcWriter.append(path)
    with w:
        if cfg.single_file:
            idx = w.numrecs
            w.write_record("time", idx, np.float64(sim.time))
            for k in fields:
                w.write_record(k, idx, data[k])
        else:
            w.write("time", np.array([sim.time], dtype=np.float64))
            for k in fields:
                w.write(k, data[k])
    cfg.prev_output_time = sim.time
    cfg.output_count += 1
    return True
